// Blosc chunk codec for the Zarr reader and writer (host code).
//
// PetaKit5D writes Zarr chunks with blosc by default (io/cpp-zarr/src/zarr.cpp:17: cname "lz4",
// clevel 5, shuffle 1; written by blosc_compress_ctx, parallelwritezarr.cpp:339-345) and reads them
// with blosc2_decompress (parallelreadzarr.cpp:150-157).  No blosc library is in this image, so the
// container is implemented here from the published blosc chunk format:
//
//   header, 16 bytes: version, codec format version, flags, typesize, then little-endian uint32
//     nbytes (uncompressed), blocksize, cbytes (whole chunk, header included);
//   flags: 0x01 byte shuffle, 0x02 stored uncompressed after the header, 0x04 bit shuffle,
//     0x10 blocks not split into typesize streams, bits 5-7 the codec
//     (0 blosclz, 1 lz4 / lz4hc, 2 snappy, 3 zlib, 4 zstd);
//   then one int32 start offset per block (blocks of `blocksize` bytes, the last one shorter), and
//   at each block its streams: the block is split into `typesize` streams when the 0x10 flag is
//   clear, typesize <= 16, blocksize / typesize >= 128 and the block is not the short last one;
//   each stream is an int32 compressed size followed by the data, stored raw when that size equals
//   the stream's uncompressed size; the byte shuffle, when flagged, was applied per block
//   (byte j of element i at j * (bytes / typesize) + i, trailing bytes unshuffled).
//
// Codecs: lz4 (the LZ4 block format, decoded and encoded here from its published specification),
// zlib (zlib itself) and zstd (the system libzstd, loaded at run time).  blosclz, snappy, bit
// shuffle and blosc2's extended headers are refused with a message naming them.
#include <dlfcn.h>
#include <zlib.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pk_internal.h"

namespace {

uint32_t rd32(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24); }
void wr32(uint8_t* p, uint32_t v) {
    p[0] = (uint8_t)v;
    p[1] = (uint8_t)(v >> 8);
    p[2] = (uint8_t)(v >> 16);
    p[3] = (uint8_t)(v >> 24);
}

// ---- LZ4 block format: sequences of [token][literal length +][literals][offset, 2 bytes LE][match
// length +]; token high nibble = literal length, low nibble = match length - 4, 15 = more bytes
// follow (each added, until one below 255); the last sequence has literals only.

// Decodes an LZ4 block into exactly `n` bytes; false on any malformed or overrunning input.
bool lz4_decode(const uint8_t* src, size_t slen, uint8_t* dst, size_t n) {
    size_t ip = 0, op = 0;
    while (ip < slen) {
        const unsigned token = src[ip++];
        size_t lit = token >> 4;
        if (lit == 15) {
            unsigned b;
            do {
                if (ip >= slen) return false;
                b = src[ip++];
                lit += b;
            } while (b == 255);
        }
        if (lit > slen - ip || lit > n - op) return false;
        memcpy(dst + op, src + ip, lit);
        ip += lit;
        op += lit;
        if (ip == slen) break;   // the last sequence: literals only
        if (slen - ip < 2) return false;
        const size_t off = (size_t)src[ip] | ((size_t)src[ip + 1] << 8);
        ip += 2;
        if (off == 0 || off > op) return false;
        size_t ml = (token & 15) + 4;
        if ((token & 15) == 15) {
            unsigned b;
            do {
                if (ip >= slen) return false;
                b = src[ip++];
                ml += b;
            } while (b == 255);
        }
        if (ml > n - op) return false;
        const uint8_t* m = dst + op - off;
        if (off >= ml) memcpy(dst + op, m, ml);
        else
            for (size_t i = 0; i < ml; i++) dst[op + i] = m[i];   // overlapping copy: byte by byte
        op += ml;
    }
    return op == n;
}

size_t lz4_bound(size_t n) { return n + n / 255 + 16; }

void lz4_len(std::vector<uint8_t>& o, size_t v) {   // the 255-run of a length of 15 or more
    v -= 15;
    while (v >= 255) {
        o.push_back(255);
        v -= 255;
    }
    o.push_back((uint8_t)v);
}

// Greedy LZ4 block encoder (hash of 4 bytes, 4096 entries).  Keeps the format's end rules: no match
// starts in the last 12 bytes, the last 5 bytes are literals.
void lz4_encode(const uint8_t* src, size_t n, std::vector<uint8_t>& o) {
    o.clear();
    o.reserve(lz4_bound(n));
    std::vector<uint32_t> table(4096, 0xffffffffu);
    size_t anchor = 0, ip = 0;
    const size_t mflimit = n > 12 ? n - 12 : 0;
    auto hash = [&](size_t p) {
        uint32_t v;
        memcpy(&v, src + p, 4);
        return (v * 2654435761u) >> 20;
    };
    auto emit = [&](size_t lit_from, size_t lit_len, size_t off, size_t mlen) {
        const size_t ml = mlen ? mlen - 4 : 0;
        o.push_back((uint8_t)(((lit_len >= 15 ? 15 : lit_len) << 4) | (mlen ? (ml >= 15 ? 15 : ml) : 0)));
        if (lit_len >= 15) lz4_len(o, lit_len);
        o.insert(o.end(), src + lit_from, src + lit_from + lit_len);
        if (mlen) {
            o.push_back((uint8_t)off);
            o.push_back((uint8_t)(off >> 8));
            if (ml >= 15) lz4_len(o, ml);
        }
    };
    while (n >= 13 && ip < mflimit) {
        const uint32_t h = hash(ip);
        const uint32_t cand = table[h];
        table[h] = (uint32_t)ip;
        if (cand != 0xffffffffu && ip - cand <= 65535 && memcmp(src + cand, src + ip, 4) == 0) {
            size_t len = 4;
            const size_t lim = n - 5;   // the match ends before the last 5 bytes
            while (ip + len < lim && src[cand + len] == src[ip + len]) len++;
            emit(anchor, ip - anchor, ip - cand, len);
            ip += len;
            anchor = ip;
        } else {
            ip++;
        }
    }
    emit(anchor, n - anchor, 0, 0);
}

// ---- zstd from the system library (ZSTD_compress / ZSTD_decompress), loaded on first use
struct Zstd {
    size_t (*compress)(void*, size_t, const void*, size_t, int) = nullptr;
    size_t (*decompress)(void*, size_t, const void*, size_t) = nullptr;
    size_t (*bound)(size_t) = nullptr;
    unsigned (*is_error)(size_t) = nullptr;
    bool ok = false;
};

const Zstd& zstd() {
    static Zstd z;
    static std::once_flag once;
    std::call_once(once, [] {
        void* h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
        if (!h) h = dlopen("libzstd.so", RTLD_NOW | RTLD_LOCAL);
        if (!h) return;
        z.compress = (size_t(*)(void*, size_t, const void*, size_t, int))dlsym(h, "ZSTD_compress");
        z.decompress = (size_t(*)(void*, size_t, const void*, size_t))dlsym(h, "ZSTD_decompress");
        z.bound = (size_t(*)(size_t))dlsym(h, "ZSTD_compressBound");
        z.is_error = (unsigned (*)(size_t))dlsym(h, "ZSTD_isError");
        z.ok = z.compress && z.decompress && z.bound && z.is_error;
    });
    return z;
}

enum { CODEC_BLOSCLZ = 0, CODEC_LZ4 = 1, CODEC_SNAPPY = 2, CODEC_ZLIB = 3, CODEC_ZSTD = 4 };

const char* codec_name(int c) {
    static const char* n[] = {"blosclz", "lz4", "snappy", "zlib", "zstd", "codec 5", "codec 6", "codec 7"};
    return n[c & 7];
}

bool stream_decode(int codec, const uint8_t* s, size_t sl, uint8_t* d, size_t n, std::string* err) {
    switch (codec) {
        case CODEC_LZ4:
            return lz4_decode(s, sl, d, n);
        case CODEC_ZLIB: {
            uLongf dl = (uLongf)n;
            return uncompress(d, &dl, s, (uLong)sl) == Z_OK && dl == n;
        }
        case CODEC_ZSTD: {
            const Zstd& z = zstd();
            if (!z.ok) {
                *err = "blosc: zstd chunks need libzstd.so.1, which could not be loaded";
                return false;
            }
            const size_t r = z.decompress(d, n, s, sl);
            return !z.is_error(r) && r == n;
        }
        default:
            *err = std::string("blosc: the ") + codec_name(codec) + " codec is not supported (lz4, zlib and zstd are)";
            return false;
    }
}

bool stream_encode(int codec, int clevel, const uint8_t* s, size_t n, std::vector<uint8_t>& o, std::string* err) {
    switch (codec) {
        case CODEC_LZ4:
            lz4_encode(s, n, o);
            return true;
        case CODEC_ZLIB: {
            uLongf cl = compressBound((uLong)n);
            o.resize(cl);
            if (compress2(o.data(), &cl, s, (uLong)n, std::max(1, std::min(9, clevel))) != Z_OK) return false;
            o.resize(cl);
            return true;
        }
        case CODEC_ZSTD: {
            const Zstd& z = zstd();
            if (!z.ok) {
                *err = "blosc: zstd chunks need libzstd.so.1, which could not be loaded";
                return false;
            }
            o.resize(z.bound(n));
            const size_t r = z.compress(o.data(), o.size(), s, n, std::max(1, std::min(22, clevel)));
            if (z.is_error(r)) return false;
            o.resize(r);
            return true;
        }
        default:
            *err = std::string("blosc: writing with the ") + codec_name(codec) + " codec is not supported";
            return false;
    }
}

bool split_block(bool dont_split, int typesize, size_t bsize, bool leftover) {
    return !dont_split && typesize <= 16 && typesize > 1 && bsize / typesize >= 128 && !leftover;
}

}  // namespace

// Decompresses one blosc chunk into `dst` (dst_len bytes, the chunk's uncompressed size).
bool pk_blosc_decompress(const uint8_t* src, size_t slen, uint8_t* dst, size_t dst_len, std::string* err) {
    if (slen < 16) {
        *err = "blosc: chunk shorter than its header";
        return false;
    }
    const unsigned version = src[0], flags = src[2], typesize = src[3];
    const size_t nbytes = rd32(src + 4), blocksize = rd32(src + 8), cbytes = rd32(src + 12);
    if (version == 0 || version > 4) {
        *err = "blosc: unknown format version " + std::to_string(version);
        return false;
    }
    if ((flags & 0x05) == 0x05) {   // both shuffle bits: blosc2's extended header
        *err = "blosc: blosc2 extended chunk headers are not supported";
        return false;
    }
    if (flags & 0x04) {
        *err = "blosc: bit-shuffled chunks are not supported";
        return false;
    }
    if (nbytes != dst_len || cbytes > slen || typesize == 0) {
        *err = "blosc: chunk sizes disagree with the array's chunk shape";
        return false;
    }
    if (nbytes == 0) return true;
    if (flags & 0x02) {   // stored uncompressed
        if (slen < 16 + nbytes) return false;
        memcpy(dst, src + 16, nbytes);
        return true;
    }
    if (blocksize == 0) return false;
    const int codec = flags >> 5;
    const bool doshuffle = (flags & 0x01) && typesize > 1;
    const bool dont_split = (flags & 0x10) != 0;
    const size_t nblocks = nbytes / blocksize + (nbytes % blocksize ? 1 : 0);
    if (16 + 4 * nblocks > cbytes) return false;
    std::vector<uint8_t> tmp(doshuffle ? blocksize : 0);
    for (size_t b = 0; b < nblocks; b++) {
        const bool leftover = b == nblocks - 1 && nbytes % blocksize != 0;
        const size_t bsize = leftover ? nbytes % blocksize : blocksize;
        size_t sp = rd32(src + 16 + 4 * b);
        uint8_t* out = dst + b * blocksize;
        uint8_t* work = doshuffle ? tmp.data() : out;
        const int nsplits = split_block(dont_split, (int)typesize, bsize, leftover) ? (int)typesize : 1;
        const size_t neblock = bsize / nsplits;
        for (int j = 0; j < nsplits; j++) {
            if (sp + 4 > cbytes) return false;
            const size_t cs = rd32(src + sp);
            sp += 4;
            if (cs > cbytes - sp) return false;
            if (cs == neblock) memcpy(work + j * neblock, src + sp, neblock);
            else if (!stream_decode(codec, src + sp, cs, work + j * neblock, neblock, err)) {
                if (err->empty()) *err = "blosc: corrupt " + std::string(codec_name(codec)) + " stream";
                return false;
            }
            sp += cs;
        }
        if (doshuffle) {   // undo the byte shuffle of this block
            const size_t ne = bsize / typesize;
            for (size_t i = 0; i < ne; i++)
                for (size_t k = 0; k < typesize; k++) out[i * typesize + k] = work[k * ne + i];
            memcpy(out + ne * typesize, work + ne * typesize, bsize - ne * typesize);
        }
    }
    return true;
}

// Compresses `n` bytes into one blosc chunk: byte shuffle (when shuffle and typesize > 1), blocks of
// up to 256 KB split into typesize streams (the blosc 1.x layout), each stream lz4 / zlib / zstd at
// `clevel` or stored raw when that is not smaller; the whole chunk stored uncompressed when that is
// smaller still.
bool pk_blosc_compress(const uint8_t* src, size_t n, int typesize, const std::string& cname, int clevel, bool shuffle,
                       std::vector<uint8_t>& out, std::string* err) {
    int codec;
    if (cname == "lz4" || cname == "lz4hc") codec = CODEC_LZ4;
    else if (cname == "zlib") codec = CODEC_ZLIB;
    else if (cname == "zstd") codec = CODEC_ZSTD;
    else {
        *err = "blosc: writing with cname \"" + cname + "\" is not supported (lz4, lz4hc, zlib, zstd are)";
        return false;
    }
    if (typesize < 1 || typesize > 255 || n > 0x7fffffffu - 64) {
        *err = "blosc: bad typesize or chunk larger than 2 GB";
        return false;
    }
    size_t blocksize = std::min<size_t>(n, 256 * 1024);
    if (typesize > 1 && blocksize > (size_t)typesize) blocksize -= blocksize % typesize;
    if (blocksize == 0) blocksize = 1;
    const size_t nblocks = n == 0 ? 0 : n / blocksize + (n % blocksize ? 1 : 0);
    const bool doshuffle = shuffle && typesize > 1;
    unsigned flags = (unsigned)(codec << 5) | (doshuffle ? 0x01u : 0u);
    out.assign(16 + 4 * nblocks, 0);
    std::vector<uint8_t> work(blocksize), cs;
    for (size_t b = 0; b < nblocks; b++) {
        const bool leftover = b == nblocks - 1 && n % blocksize != 0;
        const size_t bsize = leftover ? n % blocksize : blocksize;
        const uint8_t* in = src + b * blocksize;
        if (doshuffle) {
            const size_t ne = bsize / typesize;
            for (size_t i = 0; i < ne; i++)
                for (int k = 0; k < typesize; k++) work[k * ne + i] = in[i * typesize + k];
            memcpy(work.data() + ne * typesize, in + ne * typesize, bsize - ne * typesize);
            in = work.data();
        }
        wr32(out.data() + 16 + 4 * b, (uint32_t)out.size());
        const int nsplits = split_block(false, typesize, bsize, leftover) ? typesize : 1;
        const size_t neblock = bsize / nsplits;
        for (int j = 0; j < nsplits; j++) {
            if (!stream_encode(codec, clevel, in + j * neblock, neblock, cs, err)) {
                if (err->empty()) *err = "blosc: compression failed";
                return false;
            }
            const bool raw = cs.size() >= neblock;
            const size_t len = raw ? neblock : cs.size();
            uint8_t hdr[4];
            wr32(hdr, (uint32_t)len);
            out.insert(out.end(), hdr, hdr + 4);
            if (raw) out.insert(out.end(), in + j * neblock, in + (j + 1) * neblock);
            else out.insert(out.end(), cs.begin(), cs.end());
        }
    }
    if (out.size() >= n + 16) {   // not worth it: the bytes after the header, as they are
        out.assign(16, 0);
        out.insert(out.end(), src, src + n);
        flags |= 0x02;
    }
    out[0] = 2;   // format version of blosc 1.x chunks
    out[1] = 1;   // codec format version
    out[2] = (uint8_t)flags;
    out[3] = (uint8_t)typesize;
    wr32(out.data() + 4, (uint32_t)n);
    wr32(out.data() + 8, (uint32_t)blocksize);
    wr32(out.data() + 12, (uint32_t)out.size());
    return true;
}
