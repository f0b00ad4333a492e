// Zarr (v2) volumes either side of the deconvolution: the reference's readzarr / writezarr
// (io/readzarr.m, io/writezarr.m over io/cpp-zarr/src/parallelreadzarr.cpp, parallelwritezarr.cpp),
// re-implemented from the Zarr v2 storage specification.
//
//   * A MATLAB array [ny nx nz] is the Zarr array of shape [ny, nx, nz] (the reference writes order
//     "F" with chunk keys "i.j.k" in the same axis order); chunks are read in either order ("F" or "C")
//     and with either key separator ("." or "/").
//   * Compressors: none, "zlib", "gzip" and "blosc" (the reference's default, cname "lz4", clevel 5,
//     shuffle 1: io/cpp-zarr/src/zarr.cpp:17) with lz4, zlib or zstd inside (csrc/blosc.cu).
//   * Reading: the chunks that meet the requested box are decoded in parallel (one task per chunk, a
//     pool of host threads) and their intersection copied into the column-major output; a missing
//     chunk file reads as fill_value.  Writing: full-size chunks (edges padded with 0), zlib level 1
//     or none, compressed in parallel.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "pk_internal.h"

bool pk_blosc_decompress(const uint8_t* src, size_t slen, uint8_t* dst, size_t dst_len, std::string* err);
bool pk_blosc_compress(const uint8_t* src, size_t n, int typesize, const std::string& cname, int clevel, bool shuffle,
                       std::vector<uint8_t>& out, std::string* err);

namespace {

struct ZMeta {
    int64_t shape[3] = {1, 1, 1}, chunks[3] = {1, 1, 1};
    int ndim = 0;
    int es = 0;                 // element bytes
    char kind = 'u';            // 'u' unsigned, 'i' signed, 'f' float
    bool big_endian = false;
    bool order_c = false;
    std::string compressor;     // "", "zlib", "gzip", "blosc", or another id (unsupported)
    std::string cname = "lz4";  // blosc: the codec inside, its level and shuffle (for writes)
    int clevel = 5, shuffle = 1;
    std::string separator = ".";
    double fill = 0.0;
};

// ---- a small reader for the .zarray JSON object (the keys this file needs)
size_t skip_ws(const std::string& s, size_t i) {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\n' || s[i] == '\r' || s[i] == '\t')) i++;
    return i;
}

// position just after the value of "key" at the top level of the object, or npos
size_t find_key(const std::string& s, const std::string& key) {
    int depth = 0;
    bool in_str = false;
    for (size_t i = 0; i < s.size(); i++) {
        const char c = s[i];
        if (in_str) {
            if (c == '\\') { i++; continue; }
            if (c == '"') in_str = false;
            continue;
        }
        if (c == '{' || c == '[') depth++;
        else if (c == '}' || c == ']') depth--;
        else if (c == '"') {
            if (depth == 1 && s.compare(i + 1, key.size(), key) == 0 && i + 1 + key.size() < s.size() &&
                s[i + 1 + key.size()] == '"') {
                size_t j = skip_ws(s, i + 2 + key.size());
                if (j < s.size() && s[j] == ':') return skip_ws(s, j + 1);
            }
            in_str = true;
        }
    }
    return std::string::npos;
}

bool read_ints(const std::string& s, size_t i, int64_t* out, int* n) {
    if (i == std::string::npos || s[i] != '[') return false;
    *n = 0;
    i++;
    while (i < s.size() && s[i] != ']') {
        i = skip_ws(s, i);
        if (s[i] == ']') break;
        char* end;
        const long long v = strtoll(s.c_str() + i, &end, 10);
        if (end == s.c_str() + i || *n >= 3) return false;
        out[(*n)++] = v;
        i = skip_ws(s, (size_t)(end - s.c_str()));
        if (s[i] == ',') i++;
    }
    return *n > 0;
}

std::string read_str(const std::string& s, size_t i) {
    if (i == std::string::npos || s[i] != '"') return std::string();
    const size_t j = s.find('"', i + 1);
    return j == std::string::npos ? std::string() : s.substr(i + 1, j - i - 1);
}

bool read_file(const std::string& path, std::vector<uint8_t>& buf) {
    const int fd = open(path.c_str(), O_RDONLY);
    if (fd < 0) return false;
    struct stat sb;
    fstat(fd, &sb);
    buf.resize((size_t)sb.st_size);
    size_t got = 0;
    while (got < buf.size()) {
        const ssize_t r = read(fd, buf.data() + got, buf.size() - got);
        if (r <= 0) break;
        got += (size_t)r;
    }
    close(fd);
    return got == buf.size();
}

bool write_file(const std::string& path, const void* p, size_t n) {
    int fd = open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0 && errno == ENOENT) {              // "/" keys: the chunk's parent folders first
        for (size_t i = path.find('/', 1); i != std::string::npos; i = path.find('/', i + 1))
            mkdir(path.substr(0, i).c_str(), 0755);
        fd = open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
    }
    if (fd < 0) return false;
    size_t done = 0;
    while (done < n) {
        const ssize_t r = write(fd, (const char*)p + done, n - done);
        if (r <= 0) break;
        done += (size_t)r;
    }
    close(fd);
    return done == n;
}

pk_status parse_meta(const char* path, ZMeta& m) {
    std::vector<uint8_t> raw;
    if (!read_file(std::string(path) + "/.zarray", raw))
        return pk_fail(PK_ERR_INVALID, std::string("zarr file ") + path + " does not exist (no .zarray)");
    const std::string s(raw.begin(), raw.end());
    int n = 0, nc = 0;
    if (!read_ints(s, find_key(s, "shape"), m.shape, &n) || !read_ints(s, find_key(s, "chunks"), m.chunks, &nc) || n != nc)
        return pk_fail(PK_ERR_INVALID, "zarr: bad shape / chunks in .zarray");
    m.ndim = n;
    for (int k = n; k < 3; k++) m.shape[k] = m.chunks[k] = 1;
    const std::string dt = read_str(s, find_key(s, "dtype"));
    if (dt.size() < 3) return pk_fail(PK_ERR_INVALID, "zarr: bad dtype");
    m.big_endian = dt[0] == '>';
    m.kind = dt[1];
    m.es = atoi(dt.c_str() + 2);
    if (m.kind == 'b' && m.es == 1) m.kind = 'u';   // "|b1" (logical masks): one byte, 0 or 1, read as uint8
    if (!((m.kind == 'u' && (m.es == 1 || m.es == 2 || m.es == 4)) || (m.kind == 'f' && (m.es == 4 || m.es == 8))))
        return pk_fail(PK_ERR_UNSUPPORTED, "zarr: dtype " + dt + " is not supported");
    m.order_c = read_str(s, find_key(s, "order")) == "C";
    const size_t sep = find_key(s, "dimension_separator");
    if (sep != std::string::npos && s[sep] == '"') m.separator = read_str(s, sep);
    const size_t ci = find_key(s, "compressor");
    if (ci != std::string::npos && s[ci] == '{') {
        const size_t ce = s.find('}', ci);
        const std::string obj = s.substr(ci, ce - ci + 1);     // the compressor object: its "id"
        m.compressor = read_str(obj, find_key(obj, "id"));
        if (m.compressor == "blosc") {
            const size_t cn = find_key(obj, "cname");
            if (cn != std::string::npos) m.cname = read_str(obj, cn);
            const size_t cl = find_key(obj, "clevel");
            if (cl != std::string::npos) m.clevel = atoi(obj.c_str() + cl);
            const size_t sh = find_key(obj, "shuffle");
            if (sh != std::string::npos) m.shuffle = atoi(obj.c_str() + sh);
        }
    }
    const size_t fi = find_key(s, "fill_value");
    if (fi != std::string::npos && s[fi] == 't') m.fill = 1.0;                     // JSON true (bool arrays)
    else if (fi != std::string::npos && s[fi] != 'n' && s[fi] != '"' && s[fi] != 'f') m.fill = strtod(s.c_str() + fi, nullptr);
    if (!m.compressor.empty() && m.compressor != "zlib" && m.compressor != "gzip" && m.compressor != "blosc")
        return pk_fail(PK_ERR_UNSUPPORTED, "zarr: compressor \"" + m.compressor +
                                               "\" is not supported here (none, zlib, gzip and blosc are)");
    return PK_OK;
}

}  // namespace

namespace {

std::string chunk_key(const ZMeta& m, const int64_t c[3]) {
    std::string k = std::to_string(c[0]);
    for (int d = 1; d < m.ndim; d++) k += m.separator + std::to_string(c[d]);
    return k;
}

// decompress one chunk file into `out` (chunk bytes); false for a corrupt file
bool decode_chunk(const ZMeta& m, const std::vector<uint8_t>& raw, std::vector<uint8_t>& out) {
    if (m.compressor.empty()) {
        if (raw.size() < out.size()) return false;
        memcpy(out.data(), raw.data(), out.size());
        return true;
    }
    if (m.compressor == "blosc") {
        std::string err;
        return pk_blosc_decompress(raw.data(), raw.size(), out.data(), out.size(), &err);
    }
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (inflateInit2(&zs, m.compressor == "gzip" ? 16 + MAX_WBITS : MAX_WBITS) != Z_OK) return false;
    zs.next_in = const_cast<Bytef*>(raw.data());
    zs.avail_in = (uInt)raw.size();
    zs.next_out = out.data();
    zs.avail_out = (uInt)out.size();
    const int r = inflate(&zs, Z_FINISH);
    inflateEnd(&zs);
    return (r == Z_STREAM_END || r == Z_BUF_ERROR) && zs.avail_out == 0;
}

void byteswap(uint8_t* p, size_t n, int es) {
    if (es == 1) return;
    for (size_t i = 0; i < n; i += es) std::reverse(p + i, p + i + es);
}

template <typename T>
void fill_value(T* p, size_t n, double v) {
    const T t = (T)v;
    for (size_t i = 0; i < n; i++) p[i] = t;
}

void fill_bytes(uint8_t* p, size_t n, const ZMeta& m) {
    if (m.fill == 0.0) { memset(p, 0, n * m.es); return; }
    if (m.kind == 'f') {
        if (m.es == 4) fill_value((float*)p, n, m.fill);
        else fill_value((double*)p, n, m.fill);
    } else if (m.es == 1) fill_value((uint8_t*)p, n, m.fill);
    else if (m.es == 2) fill_value((uint16_t*)p, n, m.fill);
    else fill_value((uint32_t*)p, n, m.fill);
}

template <typename F>
void pfor(size_t n, int threads, F&& fn) {
    std::atomic<size_t> next(0);
    std::vector<std::thread> pool;
    const int T = (int)std::min<size_t>(n, (size_t)std::max(1, threads));
    for (int t = 0; t < T; t++)
        pool.emplace_back([&, t]() {
            for (size_t i = next++; i < n; i = next++) fn(i, t);
        });
    for (auto& th : pool) th.join();
}

int nthreads(int req) {
    if (req > 0) return req;
    return (int)std::max(1u, std::min(std::thread::hardware_concurrency(), 64u));
}

bool make_dir(const std::string& p) { return mkdir(p.c_str(), 0755) == 0 || errno == EEXIST; }

// one chunk as a single zlib / gzip stream (level 1)
bool deflate_whole(const std::vector<uint8_t>& buf, bool gz, std::vector<uint8_t>& zb) {
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (deflateInit2(&zs, 1, Z_DEFLATED, gz ? 16 + MAX_WBITS : MAX_WBITS, 8, Z_DEFAULT_STRATEGY) != Z_OK) return false;
    zb.resize(deflateBound(&zs, (uLong)buf.size()));
    zs.next_in = (Bytef*)buf.data();
    zs.avail_in = (uInt)buf.size();
    zs.next_out = zb.data();
    zs.avail_out = (uInt)zb.size();
    const bool ok = deflate(&zs, Z_FINISH) == Z_STREAM_END;
    zb.resize(zb.size() - zs.avail_out);
    deflateEnd(&zs);
    return ok;
}

// raw deflate of one piece of a chunk: the last piece ends the stream (Z_FINISH); the others end
// byte-aligned by a sync flush without the final-block bit, so the pieces, each compressed without
// the others' history, concatenate into one valid deflate stream
bool deflate_piece(const uint8_t* p, size_t n, bool last, std::vector<uint8_t>& out) {
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (deflateInit2(&zs, 1, Z_DEFLATED, -MAX_WBITS, 8, Z_DEFAULT_STRATEGY) != Z_OK) return false;
    out.resize(deflateBound(&zs, (uLong)n) + 16);
    zs.next_in = (Bytef*)p;
    zs.avail_in = (uInt)n;
    zs.next_out = out.data();
    zs.avail_out = (uInt)out.size();
    const int r = deflate(&zs, last ? Z_FINISH : Z_SYNC_FLUSH);
    const bool ok = last ? r == Z_STREAM_END : (r == Z_OK && zs.avail_in == 0 && zs.avail_out > 0);
    out.resize(out.size() - zs.avail_out);
    deflateEnd(&zs);
    return ok;
}

// Writes chunks 0..ntask-1: prep(t, buf) fills chunk t's cb bytes and returns its file name.
// comp: 0 none, 1 zlib, 2 gzip (level 1).  With at least as many chunks as threads, one task per
// chunk.  With fewer (a few large chunks), each chunk's deflate is cut into 1 MB pieces compressed
// in parallel and joined behind one zlib / gzip header, the Adler-32 / CRC-32 of the pieces joined
// with zlib's adler32_combine / crc32_combine: a standard stream that every reader decodes.
// comp 3: blosc with the codec, level, shuffle and element size of `bm`, one task per chunk.
template <typename Prep>
bool write_chunks(size_t ntask, size_t cb, int comp, int T, Prep&& prep, const ZMeta* bm = nullptr) {
    std::atomic<int> err(0);
    constexpr size_t PIECE = size_t(1) << 20;
    const size_t np = comp ? std::max<size_t>(1, (cb + PIECE - 1) / PIECE) : 1;
    if (comp == 0 || comp == 3 || np == 1 || ntask >= (size_t)T) {
        std::vector<std::vector<uint8_t>> bufs(T), zbufs(T);
        pfor(ntask, T, [&](size_t t, int w) {
            if (err) return;
            std::vector<uint8_t>& buf = bufs[w];
            const std::string fn = prep(t, buf);
            bool ok;
            if (comp == 0) ok = write_file(fn, buf.data(), buf.size());
            else if (comp == 3) {
                std::string e;
                ok = bm && pk_blosc_compress(buf.data(), buf.size(), bm->es, bm->cname, bm->clevel, bm->shuffle != 0,
                                             zbufs[w], &e) &&
                     write_file(fn, zbufs[w].data(), zbufs[w].size());
            } else ok = deflate_whole(buf, comp == 2, zbufs[w]) && write_file(fn, zbufs[w].data(), zbufs[w].size());
            if (!ok) err = 1;
        });
        return !err;
    }
    std::vector<std::vector<uint8_t>> bufs(ntask), zp(ntask * np);
    std::vector<std::string> names(ntask);
    std::vector<uLong> sums(ntask * np);
    pfor(ntask, T, [&](size_t t, int) { names[t] = prep(t, bufs[t]); });
    pfor(ntask * np, T, [&](size_t q, int) {
        if (err) return;
        const size_t t = q / np, k = q % np, off = k * PIECE, n = std::min(PIECE, cb - off);
        const uint8_t* p = bufs[t].data() + off;
        sums[q] = comp == 2 ? crc32(0L, p, (uInt)n) : adler32(1L, p, (uInt)n);
        if (!deflate_piece(p, n, k + 1 == np, zp[q])) err = 1;
    });
    if (err) return false;
    pfor(ntask, T, [&](size_t t, int) {
        if (err) return;
        uLong sum = sums[t * np];
        size_t tot = 18;
        for (size_t k = 0; k < np; k++) {
            tot += zp[t * np + k].size();
            if (k) {
                const z_off_t n = (z_off_t)std::min(PIECE, cb - k * PIECE);
                sum = comp == 2 ? crc32_combine(sum, sums[t * np + k], n) : adler32_combine(sum, sums[t * np + k], n);
            }
        }
        std::vector<uint8_t> out;
        out.reserve(tot);
        if (comp == 2) {
            const uint8_t h[10] = {0x1f, 0x8b, 8, 0, 0, 0, 0, 0, 4, 3};   // deflate, no name, fastest, Unix
            out.insert(out.end(), h, h + 10);
        } else {
            out.push_back(0x78);                                            // deflate, 32 KB window
            out.push_back(0x01);                                            // fastest; header % 31 == 0
        }
        for (size_t k = 0; k < np; k++) out.insert(out.end(), zp[t * np + k].begin(), zp[t * np + k].end());
        const uint32_t s32 = (uint32_t)sum, len32 = (uint32_t)cb;
        if (comp == 2) {
            for (int i = 0; i < 4; i++) out.push_back((uint8_t)(s32 >> (8 * i)));      // CRC-32, little-endian
            for (int i = 0; i < 4; i++) out.push_back((uint8_t)(len32 >> (8 * i)));    // size mod 2^32
        } else {
            for (int i = 3; i >= 0; i--) out.push_back((uint8_t)(s32 >> (8 * i)));     // Adler-32, big-endian
        }
        if (!write_file(names[t], out.data(), out.size())) err = 1;
    });
    return !err;
}

}  // namespace


extern "C" pk_status pk_zarr_info(const char* path, int64_t dims[3], int64_t chunks[3], int32_t* bits, int32_t* is_float) {
    if (!path || !dims) return pk_fail(PK_ERR_INVALID, "NULL path/dims");
    ZMeta m;
    pk_status s = parse_meta(path, m);
    if (s != PK_OK) return s;
    for (int k = 0; k < 3; k++) {
        dims[k] = m.shape[k];
        if (chunks) chunks[k] = m.chunks[k];
    }
    if (bits) *bits = m.es * 8;
    if (is_float) *is_float = m.kind == 'f';
    return PK_OK;
}

extern "C" pk_status pk_zarr_read(const char* path, const int64_t* bbox, void* out, int64_t out_bytes, int32_t threads) {
    if (!path || !out) return pk_fail(PK_ERR_INVALID, "NULL path/out");
    ZMeta m;
    pk_status s = parse_meta(path, m);
    if (s != PK_OK) return s;
    int64_t lo[3] = {0, 0, 0}, hi[3] = {m.shape[0], m.shape[1], m.shape[2]};   // [lo, hi) 0-based
    if (bbox) {
        for (int d = 0; d < 3; d++) {
            if (bbox[d] < 1 || bbox[d + 3] > m.shape[d] || bbox[d + 3] < bbox[d])
                return pk_fail(PK_ERR_INVALID, "zarr: the bounding box is outside the array");
            lo[d] = bbox[d] - 1;
            hi[d] = bbox[d + 3];
        }
    }
    const int64_t oy = hi[0] - lo[0], ox = hi[1] - lo[1], oz = hi[2] - lo[2];
    if ((uint64_t)out_bytes < (uint64_t)(oy * ox * oz) * m.es) return pk_fail(PK_ERR_INVALID, "output buffer too small");
    int64_t c0[3], c1[3], nc[3];
    for (int d = 0; d < 3; d++) {
        c0[d] = lo[d] / m.chunks[d];
        c1[d] = (hi[d] - 1) / m.chunks[d];
        nc[d] = c1[d] - c0[d] + 1;
    }
    const size_t ntask = (size_t)(nc[0] * nc[1] * nc[2]);
    const int T = nthreads(threads);
    const size_t cn = (size_t)(m.chunks[0] * m.chunks[1] * m.chunks[2]);
    std::vector<std::vector<uint8_t>> raws(T), bufs(T);
    std::atomic<int> err(0);
    uint8_t* o = (uint8_t*)out;
    const int es = m.es;
    if (m.compressor.empty() && !m.order_c) {
        // uncompressed, order F: a z-slab of a chunk is one byte range of its file, so each chunk's
        // part of the box is cut into z-pieces (enough for every thread to have work), each read by
        // its own pread straight into a worker buffer and copied run by run along y
        const int64_t cy = m.chunks[0], cx = m.chunks[1], cz = m.chunks[2];
        const size_t S = ntask >= (size_t)T ? 1 : ((size_t)T + ntask - 1) / ntask;
        pfor(ntask * S, T, [&](size_t q, int w) {
            if (err) return;
            const size_t t = q / S, k = q % S;
            const int64_t c[3] = {c0[0] + (int64_t)(t % nc[0]), c0[1] + (int64_t)((t / nc[0]) % nc[1]),
                                  c0[2] + (int64_t)(t / (nc[0] * nc[1]))};
            int64_t a[3], b[3];
            for (int d = 0; d < 3; d++) {
                a[d] = std::max(lo[d], c[d] * m.chunks[d]);
                b[d] = std::min(hi[d], (c[d] + 1) * m.chunks[d]);
            }
            const int64_t span = (b[2] - a[2] + (int64_t)S - 1) / (int64_t)S;
            const int64_t zs = a[2] + (int64_t)k * span, ze = std::min(b[2], zs + span);
            if (zs >= ze) return;
            const size_t slab = (size_t)(cx * cy) * es, nbytes = (size_t)(ze - zs) * slab;
            std::vector<uint8_t>& buf = bufs[w];
            buf.resize(nbytes);
            const int fd = open((std::string(path) + "/" + chunk_key(m, c)).c_str(), O_RDONLY);
            if (fd >= 0) {
                struct stat sb;
                const bool whole = fstat(fd, &sb) == 0 && (uint64_t)sb.st_size >= (uint64_t)cn * es;
                size_t got = 0;
                const off_t off = (off_t)((zs - c[2] * cz) * (int64_t)slab);
                while (whole && got < nbytes) {
                    const ssize_t r = pread(fd, buf.data() + got, nbytes - got, off + (off_t)got);
                    if (r <= 0) break;
                    got += (size_t)r;
                }
                close(fd);
                if (!whole || got != nbytes) { err = 1; return; }
                if (m.big_endian) byteswap(buf.data(), nbytes, es);
            } else {
                fill_bytes(buf.data(), nbytes / es, m);                // a chunk never written: fill_value
            }
            for (int64_t z = zs; z < ze; z++)
                for (int64_t x = a[1]; x < b[1]; x++) {
                    uint8_t* dst = o + (((z - lo[2]) * ox + (x - lo[1])) * oy + (a[0] - lo[0])) * es;
                    const uint8_t* src = buf.data() + (((z - zs) * cx + (x - c[1] * cx)) * cy + (a[0] - c[0] * cy)) * es;
                    memcpy(dst, src, (size_t)(b[0] - a[0]) * es);
                }
        });
        if (err) return pk_fail(PK_ERR_INVALID, "zarr: a chunk file is corrupt or truncated");
        return PK_OK;
    }
    pfor(ntask, T, [&](size_t t, int w) {
        if (err) return;
        const int64_t c[3] = {c0[0] + (int64_t)(t % nc[0]), c0[1] + (int64_t)((t / nc[0]) % nc[1]),
                              c0[2] + (int64_t)(t / (nc[0] * nc[1]))};
        std::vector<uint8_t>& buf = bufs[w];
        buf.resize(cn * es);
        if (read_file(std::string(path) + "/" + chunk_key(m, c), raws[w])) {
            if (!decode_chunk(m, raws[w], buf)) { err = 1; return; }
            if (m.big_endian) byteswap(buf.data(), buf.size(), es);
        } else {
            fill_bytes(buf.data(), cn, m);                       // a chunk never written: fill_value
        }
        // intersection of the chunk with the box, copied run by run along y
        int64_t a[3], b[3];
        for (int d = 0; d < 3; d++) {
            a[d] = std::max(lo[d], c[d] * m.chunks[d]);
            b[d] = std::min(hi[d], (c[d] + 1) * m.chunks[d]);
        }
        const int64_t cy = m.chunks[0], cx = m.chunks[1], cz = m.chunks[2];
        for (int64_t z = a[2]; z < b[2]; z++)
            for (int64_t x = a[1]; x < b[1]; x++) {
                const int64_t lz = z - c[2] * cz, lx = x - c[1] * cx;
                uint8_t* dst = o + (((z - lo[2]) * ox + (x - lo[1])) * oy + (a[0] - lo[0])) * es;
                if (!m.order_c) {
                    const uint8_t* src = buf.data() + (((lz * cx) + lx) * cy + (a[0] - c[0] * cy)) * es;
                    memcpy(dst, src, (size_t)(b[0] - a[0]) * es);
                } else {
                    for (int64_t y = a[0]; y < b[0]; y++) {                // C order: z fastest
                        const int64_t ly = y - c[0] * cy;
                        memcpy(dst + (y - a[0]) * es, buf.data() + (((ly * cx) + lx) * cz + lz) * es, es);
                    }
                }
            }
    });
    if (err) return pk_fail(PK_ERR_INVALID, "zarr: a chunk file is corrupt or truncated");
    return PK_OK;
}

extern "C" pk_status pk_zarr_write(const char* path, const void* data, const int64_t dims[3], int32_t bits,
                                   int32_t is_float, const int64_t chunks[3], int32_t compressor, int32_t threads) {
    if (!path || !data || !dims || !chunks) return pk_fail(PK_ERR_INVALID, "NULL path/data/dims/chunks");
    if (!((!is_float && (bits == 8 || bits == 16 || bits == 32)) || (is_float && (bits == 32 || bits == 64))))
        return pk_fail(PK_ERR_INVALID, "zarr: data must be uint8/16/32, single or double");
    if (compressor < 0 || compressor > 5)
        return pk_fail(PK_ERR_INVALID, "zarr: compressor must be 0 (none), 1 (zlib), 2 (gzip), 3 (blosc lz4), 4 (blosc zstd) "
                                       "or 5 (blosc zlib)");
    int64_t ch[3];
    for (int d = 0; d < 3; d++) {
        if (dims[d] < 1 || chunks[d] < 1) return pk_fail(PK_ERR_INVALID, "zarr: sizes must be positive");
        ch[d] = std::min(chunks[d], dims[d]);                           // blockSize = min(sz, blockSize)
    }
    const std::string root(path);
    if (!make_dir(root)) return pk_fail(PK_ERR_INVALID, "zarr: cannot create " + root);
    const int es = bits / 8;
    char meta[1024];
    // blosc: the reference's defaults (clevel 5, byte shuffle) with lz4, zstd or zlib inside
    static const char* kBlosc[3] = {"lz4", "zstd", "zlib"};
    char bcomp[160];
    if (compressor >= 3)
        snprintf(bcomp, sizeof(bcomp),
                 "{\"blocksize\": 0, \"clevel\": 5, \"cname\": \"%s\", \"id\": \"blosc\", \"shuffle\": 1}",
                 kBlosc[compressor - 3]);
    const char* comp = compressor == 1 ? "{\"id\": \"zlib\", \"level\": 1}"
                       : compressor == 2 ? "{\"id\": \"gzip\", \"level\": 1}"
                       : compressor >= 3 ? bcomp
                                         : "null";
    snprintf(meta, sizeof(meta),
             "{\n    \"chunks\": [%lld, %lld, %lld],\n    \"compressor\": %s,\n    \"dimension_separator\": \".\",\n"
             "    \"dtype\": \"<%c%d\",\n    \"fill_value\": 0,\n    \"filters\": null,\n    \"order\": \"F\",\n"
             "    \"shape\": [%lld, %lld, %lld],\n    \"zarr_format\": 2\n}\n",
             (long long)ch[0], (long long)ch[1], (long long)ch[2], comp, is_float ? 'f' : 'u', es, (long long)dims[0],
             (long long)dims[1], (long long)dims[2]);
    if (!write_file(root + "/.zarray", meta, strlen(meta))) return pk_fail(PK_ERR_INVALID, "zarr: cannot write .zarray");
    int64_t nc[3];
    for (int d = 0; d < 3; d++) nc[d] = (dims[d] + ch[d] - 1) / ch[d];
    const size_t ntask = (size_t)(nc[0] * nc[1] * nc[2]);
    const size_t cn = (size_t)(ch[0] * ch[1] * ch[2]);
    const int T = nthreads(threads);
    ZMeta m;
    m.ndim = 3;
    m.es = es;
    if (compressor >= 3) {
        static const char* kB[3] = {"lz4", "zstd", "zlib"};
        m.cname = kB[compressor - 3];
        m.clevel = 5;
        m.shuffle = 1;
    }
    const uint8_t* in = (const uint8_t*)data;
    const bool ok = write_chunks(ntask, cn * es, compressor >= 3 ? 3 : compressor, T, [&](size_t t, std::vector<uint8_t>& buf) {
        const int64_t c[3] = {(int64_t)(t % nc[0]), (int64_t)((t / nc[0]) % nc[1]), (int64_t)(t / (nc[0] * nc[1]))};
        buf.assign(cn * es, 0);                                   // edge chunks padded with the fill value
        int64_t a[3], b[3];
        for (int d = 0; d < 3; d++) {
            a[d] = c[d] * ch[d];
            b[d] = std::min(dims[d], a[d] + ch[d]);
        }
        for (int64_t z = a[2]; z < b[2]; z++)
            for (int64_t x = a[1]; x < b[1]; x++)
                memcpy(buf.data() + (((z - a[2]) * ch[1] + (x - a[1])) * ch[0]) * es,
                       in + ((z * dims[1] + x) * dims[0] + a[0]) * es, (size_t)(b[0] - a[0]) * es);
        return root + "/" + chunk_key(m, c);
    }, &m);
    if (!ok) return pk_fail(PK_ERR_INVALID, "zarr: writing a chunk of " + root + " failed");
    return PK_OK;
}

extern "C" pk_status pk_zarr_write_region(const char* path, const void* data, const int64_t bbox[6], int32_t threads) {
    if (!path || !data || !bbox) return pk_fail(PK_ERR_INVALID, "NULL path/data/bbox");
    ZMeta m;
    pk_status s = parse_meta(path, m);
    if (s != PK_OK) return s;
    if (m.order_c || m.big_endian) return pk_fail(PK_ERR_UNSUPPORTED, "zarr: region writes need order F, little endian");
    int64_t lo[3], hi[3], c0[3], nc[3];
    for (int d = 0; d < 3; d++) {
        lo[d] = bbox[d] - 1;
        hi[d] = bbox[d + 3];
        if (lo[d] < 0 || hi[d] > m.shape[d] || hi[d] <= lo[d]) return pk_fail(PK_ERR_INVALID, "zarr: the region is outside the array");
        if (lo[d] % m.chunks[d] != 0 || (hi[d] % m.chunks[d] != 0 && hi[d] != m.shape[d]))
            return pk_fail(PK_ERR_INVALID, "zarr: a region write must cover whole chunks");
        c0[d] = lo[d] / m.chunks[d];
        nc[d] = (hi[d] - lo[d] + m.chunks[d] - 1) / m.chunks[d];
    }
    const int es = m.es;
    const int64_t ry = hi[0] - lo[0], rx = hi[1] - lo[1];
    const size_t cn = (size_t)(m.chunks[0] * m.chunks[1] * m.chunks[2]);
    const int T = nthreads(threads);
    const uint8_t* in = (const uint8_t*)data;
    const int comp = m.compressor.empty() ? 0 : m.compressor == "gzip" ? 2 : m.compressor == "blosc" ? 3 : 1;
    const bool ok = write_chunks((size_t)(nc[0] * nc[1] * nc[2]), cn * es, comp, T, [&](size_t t, std::vector<uint8_t>& buf) {
        const int64_t c[3] = {c0[0] + (int64_t)(t % nc[0]), c0[1] + (int64_t)((t / nc[0]) % nc[1]),
                              c0[2] + (int64_t)(t / (nc[0] * nc[1]))};
        buf.assign(cn * es, 0);
        int64_t a[3], b[3];
        for (int d = 0; d < 3; d++) {
            a[d] = c[d] * m.chunks[d];
            b[d] = std::min(hi[d], a[d] + m.chunks[d]);
        }
        for (int64_t z = a[2]; z < b[2]; z++)
            for (int64_t x = a[1]; x < b[1]; x++)
                memcpy(buf.data() + (((z - a[2]) * m.chunks[1] + (x - a[1])) * m.chunks[0]) * es,
                       in + (((z - lo[2]) * rx + (x - lo[1])) * ry + (a[0] - lo[0])) * es, (size_t)(b[0] - a[0]) * es);
        return std::string(path) + "/" + chunk_key(m, c);
    }, &m);
    if (!ok) return pk_fail(PK_ERR_INVALID, "zarr: writing a chunk failed");
    return PK_OK;
}
