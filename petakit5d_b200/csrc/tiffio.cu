// TIFF volumes either side of the deconvolution: the reference's parallelReadTiff / parallelWriteTiff
// (io/cpp-tiff/src/parallelreadtiff.cpp, parallelwritetiff.cpp; io/readtiff.m, io/writetiff.m),
// re-implemented from the TIFF 6.0 / BigTIFF format without libtiff.
//
//   * Orientation of the MEX files: a column-major MATLAB array [ny nx nz] is stored as ImageLength ny,
//     ImageWidth nx, one page (IFD) per z; reading transposes each strip into column-major order.
//   * Reading: classic TIFF and BigTIFF, either byte order, strips (not tiles), one sample per pixel,
//     8/16/32-bit integer or 32/64-bit float samples, compression none / LZW / Deflate, horizontal
//     predictor; ImageJ's single-IFD raw stacks ("images=N", uncompressed) as the MEX reader handles them.
//     Strips are decoded in parallel (one task per strip, a pool of host threads, pread on one fd).
//   * Writing: BigTIFF (the MEX writer opens with "w8"), 512-row strips, LZW (the writetiff default) or
//     none, strips compressed in parallel then written in order, IFDs after the data.
// LZW follows TIFF 6.0 section 13: 9-12 bit codes, MSB first, Clear 256 / EOI 257, the code width
// growing one code early, Clear emitted when entry 4093 has been added.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "pk_internal.h"

namespace {

// ------------------------------------------------------------------ LZW
// a worker's output arena: grows geometrically and is never zero-filled (strips are appended)
struct Arena {
    uint8_t* p = nullptr;
    size_t n = 0, cap = 0;
    Arena() = default;
    Arena(const Arena&) = delete;
    Arena& operator=(const Arena&) = delete;
    Arena(Arena&& o) noexcept : p(o.p), n(o.n), cap(o.cap) { o.p = nullptr; o.n = o.cap = 0; }
    ~Arena() { std::free(p); }
    bool ensure(size_t extra) {                       // room for n + extra bytes
        if (n + extra <= cap) return true;
        const size_t c = std::max(n + extra, cap * 2 + 4096);
        uint8_t* q = (uint8_t*)std::realloc(p, c);
        if (!q) return false;
        p = q;
        cap = c;
        return true;
    }
};

// open-addressing table of (prefix code << 8 | byte) -> code, kept by each worker thread across
// strips.  A slot is one 64-bit word, generation << 32 | key << 12 | code, so a probe is one load
// and a new table (a Clear, a new strip) only bumps the generation; the slots are wiped when the
// 12-bit generation wraps.  16384 slots for at most 3836 entries: a load factor under 1/4.
struct LzwTable {
    static constexpr int HS = 1 << 14;
    std::vector<uint64_t> slot = std::vector<uint64_t>(HS, 0ull);
    uint64_t g = 0;
    void fresh() {
        if (++g == 4096) {
            std::fill(slot.begin(), slot.end(), 0ull);
            g = 1;
        }
    }
};

// largest LZW stream of len bytes: at most one 12-bit code per input byte, a Clear every 3836 codes,
// the first Clear and EndOfInformation
size_t lzw_bound(size_t len) { return len + len / 2 + len / 1024 + 16; }

// appends the LZW stream of in[0, len) to the arena (false when it cannot grow)
bool lzw_encode(const uint8_t* in, size_t len, Arena& out, LzwTable& tb) {
    if (!out.ensure(lzw_bound(len))) return false;
    uint8_t* dst = out.p + out.n;
    uint64_t acc = 0;                                  // pending bits are its low nb bits (nb < 32)
    int nb = 0;
    auto put = [&](unsigned code, int w) {
        acc = (acc << w) | code;
        nb += w;
        if (nb >= 32) {                                // four bytes at a time, most significant first
            nb -= 32;
            const uint32_t x = (uint32_t)(acc >> nb);
            dst[0] = (uint8_t)(x >> 24);
            dst[1] = (uint8_t)(x >> 16);
            dst[2] = (uint8_t)(x >> 8);
            dst[3] = (uint8_t)x;
            dst += 4;
        }
    };
    constexpr int HS = LzwTable::HS;
    uint64_t* slot = tb.slot.data();
    tb.fresh();
    uint64_t g = tb.g;
    int width = 9;
    unsigned next = 258;
    put(256, width);
    if (len > 0) {
        unsigned w = in[0];
        for (size_t i = 1; i < len; i++) {
            const unsigned k = in[i];
            const uint32_t kk = (w << 8) | k;
            const uint64_t tag = (g << 20) | kk;         // the slot's value without its code
            uint32_t h = (kk * 2654435761u) >> 18;
            uint64_t v = slot[h];
            if ((v >> 12) == tag) { w = (unsigned)(v & 4095u); continue; }   // the usual hit: first slot
            bool found = false;
            while ((v >> 32) == g) {
                h = (h + 1) & (HS - 1);
                v = slot[h];
                if ((v >> 12) == tag) { found = true; break; }
            }
            if (found) { w = (unsigned)(v & 4095u); continue; }
            put(w, width);
            slot[h] = (tag << 12) | next;
            next++;
            if (next == 4094) {
                put(256, width);
                tb.fresh();
                g = tb.g;
                next = 258;
                width = 9;
            } else if (next > (1u << width) - 1) {
                width++;
            }
            w = k;
        }
        put(w, width);
        next++;
        if (next == 4094) {
            put(256, width);
            width = 9;
        } else if (next > (1u << width) - 1) {
            width++;
        }
    }
    put(257, width);
    while (nb >= 8) {
        nb -= 8;
        *dst++ = (uint8_t)(acc >> nb);
    }
    if (nb) *dst++ = (uint8_t)(acc << (8 - nb));
    out.n = (size_t)(dst - out.p);
    return true;
}

// Decodes at most cap bytes into out; returns the bytes written or -1 for a corrupt stream.  Every
// table string is a run of the output already written (the previous string plus the first byte
// of the next), so a code is emitted by copying that run: each entry keeps its offset and length.
long long lzw_decode(const uint8_t* in, size_t len, uint8_t* out, size_t cap) {
    uint32_t off[4096];
    uint32_t length[4096];
    size_t ip = 0, o = 0;
    uint64_t bits = 0;
    int nb = 0;
    int width = 9;
    unsigned next = 258;
    int prev = -1;
    auto get = [&](int w) -> unsigned {
        if (nb < w) {
            if (ip + 8 <= len) {                      // 6 or 7 whole bytes from one big-endian load
                uint64_t x;
                memcpy(&x, in + ip, 8);
                x = __builtin_bswap64(x);
                const int take = (63 - nb) >> 3;
                bits = (bits << (8 * take)) | (x >> (64 - 8 * take));
                ip += take;
                nb += 8 * take;
            } else {
                while (nb <= 56 && ip < len) {
                    bits = (bits << 8) | in[ip++];
                    nb += 8;
                }
                if (nb < w) return 257;               // out of input: as EndOfInformation
            }
        }
        nb -= w;
        return (unsigned)(bits >> nb) & ((1u << w) - 1);
    };
    // write string `code` at o (a literal, or a copy of its earlier run); false once the strip is full
    auto emit = [&](unsigned code) -> bool {
        if (code < 256) {
            if (o >= cap) return false;
            out[o++] = (uint8_t)code;
            return o < cap;
        }
        const size_t L = length[code];
        const uint8_t* src = out + off[code];    // the run ends at or before o
        if (L <= 16 && o + 16 <= cap) {          // one 16-byte load then store: the bytes past L lie
            uint64_t lo, hi;                     // inside the strip and later codes overwrite them
            memcpy(&lo, src, 8);
            memcpy(&hi, src + 8, 8);
            memcpy(out + o, &lo, 8);
            memcpy(out + o + 8, &hi, 8);
            o += L;
            return o < cap;
        }
        const size_t n = std::min<size_t>(L, cap - o);
        if (n <= 16) {
            for (size_t i = 0; i < n; i++) out[o + i] = src[i];
        } else {
            memcpy(out + o, src, n);
        }
        o += n;
        return n == L && o < cap;
    };
    while (true) {
        unsigned code = get(width);
        if (code == 257) break;
        if (code == 256) {
            width = 9;
            next = 258;
            prev = -1;
            continue;
        }
        const size_t start = o;
        if (prev < 0) {                            // the first code after Clear (or a stream without one)
            if (code >= 256) return -1;
            if (!emit(code)) break;
            prev = (int)code;
            continue;
        }
        const size_t plen = prev < 256 ? 1 : length[prev];
        if (code < next) {
            if (!emit(code)) {
                o = std::min(o, cap);
                break;
            }
        } else if (code == next && next < 4096) {
            // KwKwK: the previous string followed by its own first byte
            const size_t pstart = start - plen;
            const size_t n = std::min(plen, cap - o);
            memcpy(out + o, out + pstart, n);
            o += n;
            if (o >= cap) break;
            out[o++] = out[pstart];
            if (o >= cap) break;
        } else {
            return -1;
        }
        if (next < 4096) {                         // previous string + first byte of this one
            off[next] = (uint32_t)(start - plen);
            length[next] = (uint32_t)(plen + 1);
            next++;
        }
        prev = (int)code;
        if (next == (1u << width) - 1 && width < 12) width++;
    }
    return (long long)o;
}

// ------------------------------------------------------------------ file parsing
struct Page {
    uint64_t w = 0, h = 0, bits = 0, fmt = 1, comp = 1, pred = 1, spp = 1, planar = 1, rows = 0;
    std::vector<uint64_t> off, cnt;
    bool tiled = false;
    std::string desc;
};

struct TiffFile {
    int fd = -1;
    bool big = false, swap = false;
    uint64_t size = 0;
    std::vector<Page> pages;
    ~TiffFile() { if (fd >= 0) close(fd); }
    bool rd(uint64_t off, void* dst, size_t n) const {
        if (off + n > size) return false;
        size_t got = 0;
        while (got < n) {
            const ssize_t r = pread(fd, (char*)dst + got, n - got, (off_t)(off + got));
            if (r <= 0) return false;
            got += (size_t)r;
        }
        return true;
    }
    uint16_t u16(const uint8_t* p) const { uint16_t v; memcpy(&v, p, 2); return swap ? __builtin_bswap16(v) : v; }
    uint32_t u32(const uint8_t* p) const { uint32_t v; memcpy(&v, p, 4); return swap ? __builtin_bswap32(v) : v; }
    uint64_t u64(const uint8_t* p) const { uint64_t v; memcpy(&v, p, 8); return swap ? __builtin_bswap64(v) : v; }
};

int type_size(unsigned t) {
    switch (t) {
        case 1: case 2: case 6: case 7: return 1;
        case 3: case 8: return 2;
        case 4: case 9: case 11: case 13: return 4;
        case 5: case 10: case 12: case 16: case 17: case 18: return 8;
        default: return 0;
    }
}

pk_status open_tiff(const char* path, TiffFile& f) {
    f.fd = open(path, O_RDONLY);
    if (f.fd < 0) return pk_fail(PK_ERR_INVALID, std::string("File \"") + path + "\" cannot be opened");
    struct stat sb;
    fstat(f.fd, &sb);
    f.size = (uint64_t)sb.st_size;
    uint8_t hd[16];
    if (!f.rd(0, hd, 8)) return pk_fail(PK_ERR_INVALID, "not a TIFF file (short header)");
    if (hd[0] == 'I' && hd[1] == 'I') f.swap = false;
    else if (hd[0] == 'M' && hd[1] == 'M') f.swap = true;
    else return pk_fail(PK_ERR_INVALID, "not a TIFF file (byte order mark)");
    const uint16_t magic = f.u16(hd + 2);
    uint64_t ifd;
    if (magic == 42) ifd = f.u32(hd + 4);
    else if (magic == 43) {
        if (!f.rd(0, hd, 16)) return pk_fail(PK_ERR_INVALID, "short BigTIFF header");
        f.big = true;
        ifd = f.u64(hd + 8);
    } else return pk_fail(PK_ERR_INVALID, "not a TIFF file (magic)");
    const int esz = f.big ? 20 : 12, csz = f.big ? 8 : 2, osz = f.big ? 8 : 4;
    size_t guard = 0;
    while (ifd && guard++ < (1u << 24)) {
        uint8_t cb[8];
        if (!f.rd(ifd, cb, csz)) return pk_fail(PK_ERR_INVALID, "truncated IFD");
        const uint64_t n = f.big ? f.u64(cb) : f.u16(cb);
        if (n > 4096) return pk_fail(PK_ERR_INVALID, "implausible IFD entry count");
        std::vector<uint8_t> e(n * esz + osz);
        if (!f.rd(ifd + csz, e.data(), e.size())) return pk_fail(PK_ERR_INVALID, "truncated IFD");
        Page pg;
        for (uint64_t k = 0; k < n; k++) {
            const uint8_t* p = e.data() + k * esz;
            const unsigned tag = f.u16(p), typ = f.u16(p + 2);
            const uint64_t cnt = f.big ? f.u64(p + 4) : f.u32(p + 4);
            const uint8_t* fld = p + (f.big ? 12 : 8);
            const int ts = type_size(typ);
            if (!ts) continue;
            const uint64_t bytes = cnt * (uint64_t)ts;
            std::vector<uint8_t> val(bytes);
            if (bytes <= (uint64_t)osz) memcpy(val.data(), fld, bytes);
            else {
                const uint64_t vo = f.big ? f.u64(fld) : f.u32(fld);
                if (!f.rd(vo, val.data(), bytes)) return pk_fail(PK_ERR_INVALID, "tag value out of file");
            }
            auto num = [&](uint64_t i) -> uint64_t {
                const uint8_t* q = val.data() + i * ts;
                switch (ts) {
                    case 1: return q[0];
                    case 2: return f.u16(q);
                    case 4: return f.u32(q);
                    default: return f.u64(q);
                }
            };
            switch (tag) {
                case 256: pg.w = num(0); break;
                case 257: pg.h = num(0); break;
                case 258: pg.bits = num(0); break;
                case 259: pg.comp = num(0); break;
                case 270: pg.desc.assign((const char*)val.data(), bytes); break;
                case 273: pg.off.resize(cnt); for (uint64_t i = 0; i < cnt; i++) pg.off[i] = num(i); break;
                case 277: pg.spp = num(0); break;
                case 278: pg.rows = num(0); break;
                case 279: pg.cnt.resize(cnt); for (uint64_t i = 0; i < cnt; i++) pg.cnt[i] = num(i); break;
                case 284: pg.planar = num(0); break;
                case 317: pg.pred = num(0); break;
                case 322: case 323: case 324: case 325: pg.tiled = true; break;
                case 339: pg.fmt = num(0); break;
                default: break;
            }
        }
        if (!pg.rows || pg.rows > pg.h) pg.rows = pg.h;
        f.pages.push_back(std::move(pg));
        const uint8_t* np = e.data() + n * esz;
        ifd = f.big ? f.u64(np) : f.u32(np);
    }
    if (f.pages.empty()) return pk_fail(PK_ERR_INVALID, "TIFF without images");
    return PK_OK;
}

// ImageJ raw stack: one IFD, uncompressed, "images=N" in ImageDescription (the MEX reader's isImageJIm)
uint64_t imagej_images(const TiffFile& f) {
    if (f.pages.size() != 1) return 0;
    const Page& p = f.pages[0];
    if (p.comp != 1 || p.desc.find("ImageJ") == std::string::npos) return 0;
    const size_t k = p.desc.find("images=");
    if (k == std::string::npos) return 0;
    return strtoull(p.desc.c_str() + k + 7, nullptr, 10);
}

pk_status check_page(const Page& p, const Page& p0) {
    if (p.tiled) return pk_fail(PK_ERR_UNSUPPORTED, "tiled TIFF images are not supported");
    if (p.spp != 1 || p.planar != 1) return pk_fail(PK_ERR_UNSUPPORTED, "only one sample per pixel is supported");
    if (p.w != p0.w || p.h != p0.h || p.bits != p0.bits || p.fmt != p0.fmt)
        return pk_fail(PK_ERR_INVALID, "TIFF pages differ in size or sample type");
    if (p.comp != 1 && p.comp != 5 && p.comp != 8 && p.comp != 32946)
        return pk_fail(PK_ERR_UNSUPPORTED, "TIFF compression " + std::to_string(p.comp) + " is not supported");
    if (p.pred != 1 && p.pred != 2) return pk_fail(PK_ERR_UNSUPPORTED, "TIFF predictor " + std::to_string(p.pred) + " is not supported");
    if (p.pred == 2 && p.fmt == 3) return pk_fail(PK_ERR_UNSUPPORTED, "horizontal predictor on float samples");
    const uint64_t ns = (p.h + p.rows - 1) / p.rows;
    if (p.off.size() < ns || p.cnt.size() < ns) return pk_fail(PK_ERR_INVALID, "missing strip offsets");
    return PK_OK;
}

template <typename T>
void undo_predictor(T* row, uint64_t w) {
    for (uint64_t i = 1; i < w; i++) row[i] = (T)(row[i] + row[i - 1]);
}

void swap_bytes(uint8_t* p, size_t n, int es) {
    if (es == 2) for (size_t i = 0; i < n; i += 2) std::swap(p[i], p[i + 1]);
    else if (es == 4) for (size_t i = 0; i < n; i += 4) { std::swap(p[i], p[i + 3]); std::swap(p[i + 1], p[i + 2]); }
    else if (es == 8) for (size_t i = 0; i < n; i += 8) for (int k = 0; k < 4; k++) std::swap(p[i + k], p[i + 7 - k]);
}

// d[j * ds + i] = s[i * ss + j] for an 8 x 8 block of 16-bit values: three rounds of interleaves
// (SSE2, part of every x86-64 CPU), or plain loads and stores elsewhere
inline void transpose8x8_u16(const uint16_t* s, uint64_t ss, uint16_t* d, uint64_t ds) {
#if defined(__SSE2__)
    __m128i a[8], b[8], c[8];
    for (int i = 0; i < 8; i++) a[i] = _mm_loadu_si128((const __m128i*)(s + i * ss));
    for (int i = 0; i < 4; i++) {
        b[2 * i] = _mm_unpacklo_epi16(a[2 * i], a[2 * i + 1]);      // rows 2i, 2i+1: columns 0-3
        b[2 * i + 1] = _mm_unpackhi_epi16(a[2 * i], a[2 * i + 1]);  // columns 4-7
    }
    for (int i = 0; i < 2; i++) {
        c[4 * i + 0] = _mm_unpacklo_epi32(b[4 * i + 0], b[4 * i + 2]);   // rows 4i..4i+3: columns 0, 1
        c[4 * i + 1] = _mm_unpackhi_epi32(b[4 * i + 0], b[4 * i + 2]);   // columns 2, 3
        c[4 * i + 2] = _mm_unpacklo_epi32(b[4 * i + 1], b[4 * i + 3]);   // columns 4, 5
        c[4 * i + 3] = _mm_unpackhi_epi32(b[4 * i + 1], b[4 * i + 3]);   // columns 6, 7
    }
    for (int j = 0; j < 4; j++) {
        _mm_storeu_si128((__m128i*)(d + (2 * j) * ds), _mm_unpacklo_epi64(c[j], c[4 + j]));
        _mm_storeu_si128((__m128i*)(d + (2 * j + 1) * ds), _mm_unpackhi_epi64(c[j], c[4 + j]));
    }
#else
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) d[j * ds + i] = s[i * ss + j];
#endif
}

// Transpose of an nr x w row-major block (row stride w) into a column-major array with column
// stride h, in 32 x 32 tiles so that both sides stay in cache (whole 16-bit tiles by 8 x 8 blocks).
template <typename T>
void transpose_block(const T* src, uint64_t nr, uint64_t w, T* dst, uint64_t h) {
    constexpr uint64_t B = 32;
    for (uint64_t r0 = 0; r0 < nr; r0 += B) {
        const uint64_t r1 = std::min(nr, r0 + B);
        for (uint64_t x0 = 0; x0 < w; x0 += B) {
            const uint64_t x1 = std::min(w, x0 + B);
            if (sizeof(T) == 2 && r1 - r0 == B && x1 - x0 == B) {   // whole tile: 8 x 8 blocks
                for (uint64_t x = x0; x < x1; x += 8)
                    for (uint64_t r = r0; r < r1; r += 8)
                        transpose8x8_u16((const uint16_t*)src + r * w + x, w, (uint16_t*)dst + x * h + r, h);
                continue;
            }
            for (uint64_t x = x0; x < x1; x++) {
                const T* s = src + x;
                T* d = dst + x * h;
                for (uint64_t r = r0; r < r1; r++) d[r] = s[r * w];
            }
        }
    }
}

// rows [r0, r0 + nr) of page z (row-major, row stride w) into the column-major output [h w nz]
void scatter_rows(const uint8_t* rows, uint64_t r0, uint64_t nr, uint64_t w, uint64_t h, uint64_t z, int es, uint8_t* out) {
    const uint64_t base = z * w * h + r0;
    switch (es) {
        case 1: transpose_block((const uint8_t*)rows, nr, w, (uint8_t*)out + base, h); break;
        case 2: transpose_block((const uint16_t*)rows, nr, w, (uint16_t*)out + base, h); break;
        case 4: transpose_block((const uint32_t*)rows, nr, w, (uint32_t*)out + base, h); break;
        default: transpose_block((const uint64_t*)rows, nr, w, (uint64_t*)out + base, h); break;
    }
}

// column-major rows [r0, r0 + nr) of a plane (column stride h) into a row-major strip (row stride w)
void gather_rows(const uint8_t* plane, uint64_t r0, uint64_t nr, uint64_t w, uint64_t h, int es, uint8_t* rows) {
    auto go = [&](auto tag) {
        using T = decltype(tag);
        const T* src = (const T*)plane + r0;
        T* dst = (T*)rows;
        constexpr uint64_t B = 32;
        for (uint64_t x0 = 0; x0 < w; x0 += B) {
            const uint64_t x1 = std::min(w, x0 + B);
            for (uint64_t q0 = 0; q0 < nr; q0 += B) {
                const uint64_t q1 = std::min(nr, q0 + B);
                if (sizeof(T) == 2 && x1 - x0 == B && q1 - q0 == B) {  // whole tile: 8 x 8 blocks
                    for (uint64_t x = x0; x < x1; x += 8)
                        for (uint64_t r = q0; r < q1; r += 8)
                            transpose8x8_u16((const uint16_t*)src + x * h + r, h, (uint16_t*)dst + r * w + x, w);
                    continue;
                }
                for (uint64_t x = x0; x < x1; x++)
                    for (uint64_t r = q0; r < q1; r++) dst[r * w + x] = src[x * h + r];
            }
        }
    };
    switch (es) {
        case 1: go(uint8_t()); break;
        case 2: go(uint16_t()); break;
        case 4: go(uint32_t()); break;
        default: go(uint64_t()); break;
    }
}

int n_threads(int req) {
    if (req > 0) return req;
    const unsigned hc = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(hc, 64u));
}

// fn(task, worker): tasks handed out in order to `threads` workers (a worker index lets each keep
// its buffers across tasks instead of allocating per strip)
template <typename F>
void parallel_for(size_t n, int threads, F&& fn) {
    std::atomic<size_t> next(0);
    std::vector<std::thread> pool;
    const int T = (int)std::min<size_t>(n, (size_t)threads);
    for (int t = 0; t < T; t++)
        pool.emplace_back([&, t]() {
            for (size_t i = next++; i < n; i = next++) fn(i, t);
        });
    for (auto& th : pool) th.join();
}

// ------------------------------------------------------------------ writing
struct Out {
    int fd;
    std::atomic<bool> ok{true};
    void put(uint64_t off, const void* p, size_t n) {
        size_t done = 0;
        while (ok.load(std::memory_order_relaxed) && done < n) {
            const ssize_t r = pwrite(fd, (const char*)p + done, n - done, (off_t)(off + done));
            if (r <= 0) ok = false;
            else done += (size_t)r;
        }
    }
};

}  // namespace

extern "C" pk_status pk_tiff_info(const char* path, int64_t dims[3], int32_t* bits, int32_t* is_float) {
    if (!path || !dims) return pk_fail(PK_ERR_INVALID, "NULL path/dims");
    TiffFile f;
    pk_status s;
    if ((s = open_tiff(path, f)) != PK_OK) return s;
    const Page& p = f.pages[0];
    const uint64_t ij = imagej_images(f);
    dims[0] = (int64_t)p.h;
    dims[1] = (int64_t)p.w;
    dims[2] = (int64_t)(ij ? ij : f.pages.size());
    if (bits) *bits = (int32_t)p.bits;
    if (is_float) *is_float = p.fmt == 3;
    return PK_OK;
}

extern "C" pk_status pk_tiff_read(const char* path, const int64_t* z_range, void* out, int64_t out_bytes, int32_t threads) {
    if (!path || !out) return pk_fail(PK_ERR_INVALID, "NULL path/out");
    TiffFile f;
    pk_status s;
    if ((s = open_tiff(path, f)) != PK_OK) return s;
    const Page& p0 = f.pages[0];
    const uint64_t ij = imagej_images(f);
    const uint64_t nz = ij ? ij : f.pages.size();
    uint64_t z0 = 0, z1 = nz;
    if (z_range) {
        if (z_range[0] < 1 || z_range[1] < z_range[0] || (uint64_t)z_range[1] > nz)
            return pk_fail(PK_ERR_INVALID, "Range is out of bounds");
        z0 = (uint64_t)z_range[0] - 1;
        z1 = (uint64_t)z_range[1];
    }
    if (p0.bits != 8 && p0.bits != 16 && p0.bits != 32 && p0.bits != 64)
        return pk_fail(PK_ERR_UNSUPPORTED, "Data type not suppported (bits per sample " + std::to_string(p0.bits) + ")");
    const int es = (int)(p0.bits / 8);
    const uint64_t w = p0.w, h = p0.h;
    const uint64_t need = w * h * (z1 - z0) * es;
    if ((uint64_t)out_bytes < need) return pk_fail(PK_ERR_INVALID, "output buffer too small");
    const int T = n_threads(threads);
    std::atomic<int> err(0);
    if (ij) {
        if ((s = check_page(p0, p0)) != PK_OK) return s;
        const uint64_t pb = w * h * es, base = p0.off[0];
        std::vector<std::vector<uint8_t>> pages(T);
        parallel_for(z1 - z0, T, [&](size_t k, int t) {
            std::vector<uint8_t>& page = pages[t];
            page.resize(pb);
            if (!f.rd(base + (z0 + k) * pb, page.data(), pb)) { err = 1; return; }
            if (f.swap && es > 1) swap_bytes(page.data(), pb, es);
            scatter_rows(page.data(), 0, h, w, h, k, es, (uint8_t*)out);
        });
        if (err) return pk_fail(PK_ERR_INVALID, "ImageJ stack extends past the end of the file");
        return PK_OK;
    }
    for (uint64_t z = z0; z < z1; z++)
        if ((s = check_page(f.pages[z], p0)) != PK_OK) return s;
    // one task per strip
    std::vector<std::pair<uint64_t, uint64_t>> tasks;
    for (uint64_t z = z0; z < z1; z++) {
        const uint64_t ns = (h + f.pages[z].rows - 1) / f.pages[z].rows;
        for (uint64_t k = 0; k < ns; k++) tasks.push_back({z, k});
    }
    std::vector<std::vector<uint8_t>> raws(T), rowss(T);
    parallel_for(tasks.size(), T, [&](size_t t, int worker) {
        if (err) return;
        const uint64_t z = tasks[t].first, k = tasks[t].second;
        const Page& p = f.pages[z];
        const uint64_t r0 = k * p.rows, nr = std::min(p.rows, h - r0);
        const uint64_t want = nr * w * es;
        std::vector<uint8_t>& raw = raws[worker];
        std::vector<uint8_t>& rows = rowss[worker];
        raw.resize(p.cnt[k]);
        rows.resize(want);
        if (!f.rd(p.off[k], raw.data(), raw.size())) { err = 2; return; }
        if (p.comp == 1) {
            if (raw.size() < want) { err = 2; return; }
            memcpy(rows.data(), raw.data(), want);
        } else if (p.comp == 5) {
            const long long got = lzw_decode(raw.data(), raw.size(), rows.data(), want);
            if (got < 0) { err = 3; return; }
            if ((uint64_t)got < want) memset(rows.data() + got, 0, want - got);
        } else {
            uLongf dl = (uLongf)want;
            const int zr = uncompress(rows.data(), &dl, raw.data(), (uLong)raw.size());
            if (zr != Z_OK && zr != Z_BUF_ERROR) { err = 3; return; }
        }
        if (f.swap && es > 1) swap_bytes(rows.data(), want, es);
        if (p.pred == 2)
            for (uint64_t r = 0; r < nr; r++) {
                uint8_t* row = rows.data() + r * w * es;
                if (es == 1) undo_predictor((uint8_t*)row, w);
                else if (es == 2) undo_predictor((uint16_t*)row, w);
                else if (es == 4) undo_predictor((uint32_t*)row, w);
                else undo_predictor((uint64_t*)row, w);
            }
        scatter_rows(rows.data(), r0, nr, w, h, z - z0, es, (uint8_t*)out);
    });
    if (err == 2) return pk_fail(PK_ERR_INVALID, "strip data past the end of the file");
    if (err == 3) return pk_fail(PK_ERR_INVALID, "corrupt compressed strip");
    return PK_OK;
}

extern "C" pk_status pk_tiff_write(const char* path, const void* data, const int64_t dims[3], int32_t bits,
                                   int32_t is_float, int32_t lzw, int32_t threads) {
    if (!path || !data || !dims) return pk_fail(PK_ERR_INVALID, "NULL path/data/dims");
    if (bits != 8 && bits != 16 && bits != 32 && bits != 64) return pk_fail(PK_ERR_INVALID, "bits must be 8, 16, 32 or 64");
    if (is_float && bits < 32) return pk_fail(PK_ERR_INVALID, "float samples are 32 or 64 bits");
    const uint64_t h = (uint64_t)dims[0], w = (uint64_t)dims[1], nz = dims[2] > 0 ? (uint64_t)dims[2] : 1;
    if (!h || !w) return pk_fail(PK_ERR_INVALID, "All input data axes must be of at least size 1");
    const int es = bits / 8;
    const uint64_t rps = 512, ns = (h + rps - 1) / rps;
    // strips: transpose the column-major plane rows into row-major strips, compress in parallel
    // each worker appends its strips to an arena of its own (no allocation per strip)
    const int T = (int)std::min<uint64_t>(nz * ns, (uint64_t)n_threads(threads));
    std::vector<Arena> arena(T);
    std::vector<std::vector<uint8_t>> rowss(T);
    std::vector<LzwTable> tables(lzw ? T : 0);
    struct StripRef { int worker; size_t off, size; };
    std::vector<StripRef> strips(nz * ns);
    std::atomic<bool> grown(true);
    parallel_for(nz * ns, T, [&](size_t t, int worker) {
        const uint64_t z = t / ns, k = t % ns, r0 = k * rps, nr = std::min(rps, h - r0);
        Arena& a = arena[worker];
        const size_t at = a.n;
        const uint8_t* plane = (const uint8_t*)data + z * w * h * es;
        if (lzw) {
            std::vector<uint8_t>& rows = rowss[worker];
            rows.resize(nr * w * es);
            gather_rows(plane, r0, nr, w, h, es, rows.data());
            if (!lzw_encode(rows.data(), rows.size(), a, tables[worker])) grown = false;
        } else if (a.ensure(nr * w * es)) {
            gather_rows(plane, r0, nr, w, h, es, a.p + at);
            a.n += nr * w * es;
        } else {
            grown = false;
        }
        strips[t] = {worker, at, a.n - at};
    });
    if (!grown) return pk_fail(PK_ERR_NOMEM, "out of host memory for the compressed strips");
    const int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) return pk_fail(PK_ERR_INVALID, std::string("cannot create \"") + path + "\"");
    Out o{fd};
    // strip offsets by a prefix sum, then the strips written in parallel at their offsets
    std::vector<uint64_t> soff(nz * ns);
    uint64_t pos = 16;
    for (size_t t = 0; t < strips.size(); t++) {
        soff[t] = pos;
        pos += strips[t].size;
    }
    parallel_for(strips.size(), T, [&](size_t t, int) {
        o.put(soff[t], arena[strips[t].worker].p + strips[t].off, strips[t].size);
    });
    pos = (pos + 7) & ~7ull;
    const uint64_t first_ifd = pos;
    // IFDs: 11 entries; strip offsets / byte counts out of line when more than one strip; all of
    // them assembled in one buffer and written at once
    const int NE = 11;
    const uint64_t ifd_bytes = 8 + NE * 20 + 8 + (ns > 1 ? 16 * ns : 0);
    std::vector<uint8_t> ifds(nz * ifd_bytes, 0);
    for (uint64_t z = 0; z < nz; z++) {
        const uint64_t ifd = first_ifd + z * ifd_bytes, arr = ifd + 8 + NE * 20 + 8;
        const uint64_t next = z + 1 < nz ? ifd + ifd_bytes : 0;
        uint8_t* b = ifds.data() + z * ifd_bytes;
        uint64_t n = NE;
        memcpy(b, &n, 8);
        uint8_t* e = b + 8;
        auto ent = [&](uint16_t tag, uint16_t typ, uint64_t cnt, uint64_t val) {
            memcpy(e, &tag, 2);
            memcpy(e + 2, &typ, 2);
            memcpy(e + 4, &cnt, 8);
            memcpy(e + 12, &val, 8);
            e += 20;
        };
        ent(256, 4, 1, w);
        ent(257, 4, 1, h);
        ent(258, 3, 1, (uint64_t)bits);
        ent(259, 3, 1, lzw ? 5 : 1);
        ent(262, 3, 1, 1);
        ent(273, 16, ns, ns > 1 ? arr : soff[z * ns]);
        ent(277, 3, 1, 1);
        ent(278, 4, 1, rps);
        ent(279, 16, ns, ns > 1 ? arr + 8 * ns : strips[z * ns].size);
        ent(284, 3, 1, 1);
        ent(339, 3, 1, is_float ? 3 : 1);
        memcpy(b + 8 + NE * 20, &next, 8);
        if (ns > 1) {
            uint8_t* a = b + 8 + NE * 20 + 8;
            for (uint64_t k = 0; k < ns; k++) {
                const uint64_t off = soff[z * ns + k], cnt = strips[z * ns + k].size;
                memcpy(a + 8 * k, &off, 8);
                memcpy(a + 8 * (ns + k), &cnt, 8);
            }
        }
    }
    o.put(first_ifd, ifds.data(), ifds.size());
    const uint8_t hd[8] = {'I', 'I', 43, 0, 8, 0, 0, 0};
    o.put(0, hd, 8);
    o.put(8, &first_ifd, 8);
    const bool ok = o.ok;
    close(fd);
    if (!ok) return pk_fail(PK_ERR_INVALID, std::string("write to \"") + path + "\" failed");
    return PK_OK;
}

extern "C" pk_status pk_host_alloc(int64_t bytes, void** ptr) {
    if (!ptr || bytes < 0) return pk_fail(PK_ERR_INVALID, "bad host allocation request");
    const cudaError_t e = cudaHostAlloc(ptr, (size_t)std::max<int64_t>(bytes, 1), cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        return pk_fail(PK_ERR_NOMEM, std::string("pinned host allocation failed: ") + cudaGetErrorString(e));
    }
    return PK_OK;
}

extern "C" pk_status pk_host_free(void* ptr) {
    if (ptr && cudaFreeHost(ptr) != cudaSuccess) {
        cudaGetLastError();
        return pk_fail(PK_ERR_INVALID, "not a pinned host allocation");
    }
    return PK_OK;
}
