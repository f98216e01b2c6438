// .npy / .npz reader (own implementation of the published NPY format and the
// ZIP container with ZIP64 extensions; deflate through zlib).
#include "dtb_io.h"

#include <algorithm>

#include <zlib.h>

#include <cstdio>
#include <cstring>

namespace dtb {

int NpyArray::item_size() const
{
    if (descr.size() < 3) return 0;
    return std::atoi(descr.c_str() + 2);
}

static uint16_t rd16(const unsigned char* p) { return (uint16_t)(p[0] | (p[1] << 8)); }
static uint32_t rd32(const unsigned char* p)
{
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static uint64_t rd64(const unsigned char* p) { return (uint64_t)rd32(p) | ((uint64_t)rd32(p + 4) << 32); }

static std::string dict_value(const std::string& h, const std::string& key)
{
    size_t k = h.find("'" + key + "'");
    if (k == std::string::npos) return "";
    size_t c = h.find(':', k);
    if (c == std::string::npos) return "";
    size_t s = c + 1;
    while (s < h.size() && h[s] == ' ') ++s;
    if (s >= h.size()) return "";
    if (h[s] == '\'') {
        size_t e = h.find('\'', s + 1);
        return e == std::string::npos ? "" : h.substr(s + 1, e - s - 1);
    }
    if (h[s] == '(') {
        size_t e = h.find(')', s);
        return e == std::string::npos ? "" : h.substr(s, e - s + 1);
    }
    size_t e = s;
    while (e < h.size() && h[e] != ',' && h[e] != '}') ++e;
    return h.substr(s, e - s);
}

bool npy_parse(const char* buf, size_t len, NpyArray& out, std::string& err)
{
    const unsigned char* p = reinterpret_cast<const unsigned char*>(buf);
    if (len < 10 || std::memcmp(p, "\x93NUMPY", 6) != 0) { err = "not an .npy buffer"; return false; }
    const int major = p[6];
    size_t hlen, off;
    if (major == 1) { hlen = rd16(p + 8); off = 10; }
    else { if (len < 12) { err = "truncated .npy header"; return false; } hlen = rd32(p + 8); off = 12; }
    if (off + hlen > len) { err = "truncated .npy header"; return false; }
    std::string h(buf + off, hlen);
    out.descr = dict_value(h, "descr");
    out.fortran = dict_value(h, "fortran_order").find("True") != std::string::npos;
    std::string shp = dict_value(h, "shape");
    out.shape.clear();
    if (out.descr.empty() || shp.empty()) { err = "bad .npy header: " + h; return false; }
    for (size_t i = 1; i < shp.size();) {
        while (i < shp.size() && (shp[i] == ' ' || shp[i] == ',')) ++i;
        if (i >= shp.size() || shp[i] == ')') break;
        char* end = nullptr;
        long long v = std::strtoll(shp.c_str() + i, &end, 10);
        if (end == shp.c_str() + i) { err = "bad shape " + shp; return false; }
        out.shape.push_back(v);
        i = (size_t)(end - shp.c_str());
    }
    if (out.descr[0] == '>' && out.item_size() > 1) { err = "big-endian arrays are not supported"; return false; }
    const size_t nbytes = (size_t)out.count() * (size_t)out.item_size();
    if (off + hlen + nbytes > len) { err = "truncated .npy data"; return false; }
    out.data.assign(buf + off + hlen, buf + off + hlen + nbytes);
    return true;
}

static bool inflate_raw(const unsigned char* src, size_t n, std::vector<char>& dst, size_t expect, std::string& err)
{
    dst.resize(expect);
    z_stream zs;
    std::memset(&zs, 0, sizeof(zs));
    if (inflateInit2(&zs, -MAX_WBITS) != Z_OK) { err = "inflateInit2 failed"; return false; }
    size_t in_done = 0, out_done = 0;
    int rc = Z_OK;
    while (rc != Z_STREAM_END) {
        const size_t in_chunk = std::min<size_t>(n - in_done, 1u << 30);
        const size_t out_chunk = std::min<size_t>(expect - out_done, 1u << 30);
        zs.next_in = const_cast<unsigned char*>(src + in_done);
        zs.avail_in = (uInt)in_chunk;
        zs.next_out = reinterpret_cast<unsigned char*>(dst.data() + out_done);
        zs.avail_out = (uInt)out_chunk;
        rc = inflate(&zs, Z_NO_FLUSH);
        in_done += in_chunk - zs.avail_in;
        out_done += out_chunk - zs.avail_out;
        if (rc != Z_OK && rc != Z_STREAM_END) { inflateEnd(&zs); err = "deflate stream error"; return false; }
        if (rc == Z_OK && zs.avail_in == 0 && in_done >= n && out_done < expect) {
            inflateEnd(&zs); err = "truncated deflate stream"; return false;
        }
        if (out_done >= expect && rc != Z_STREAM_END && in_done >= n) break;
    }
    inflateEnd(&zs);
    if (out_done != expect) { err = "deflate size mismatch"; return false; }
    return true;
}

// Reads [off, off + n) of f into dst; false on a short read.
static bool read_at(FILE* f, uint64_t off, size_t n, void* dst)
{
    if (fseeko(f, (off_t)off, SEEK_SET) != 0) return false;
    return n == 0 || std::fread(dst, 1, n, f) == n;
}

bool npz_read(const std::string& path, std::map<std::string, NpyArray>& out, std::string& err,
              const std::vector<std::string>* only, std::vector<std::string>* names)
{
    // Only the archive's tail, its central directory and the wanted members are read.
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) { err = "cannot open " + path; return false; }
    struct Closer { FILE* f; ~Closer() { std::fclose(f); } } closer{f};
    fseeko(f, 0, SEEK_END);
    const uint64_t fsize = (uint64_t)ftello(f);
    if (fsize < 22) { err = "file too small for a zip archive: " + path; return false; }
    // end of central directory (within the last 64 KB + its 22 bytes)
    const uint64_t tail_n = std::min<uint64_t>(fsize, 22 + 65535 + 20);
    std::vector<unsigned char> tail((size_t)tail_n);
    if (!read_at(f, fsize - tail_n, (size_t)tail_n, tail.data())) { err = "read failed: " + path; return false; }
    long long eocd = -1;
    for (long long k = (long long)tail_n - 22; k >= 0; --k)
        if (rd32(tail.data() + k) == 0x06054b50u) { eocd = k; break; }
    if (eocd < 0) { err = "no end-of-central-directory record: " + path; return false; }
    const unsigned char* e = tail.data() + eocd;
    uint64_t n_entries = rd16(e + 10);
    uint64_t cd_size = rd32(e + 12);
    uint64_t cd_off = rd32(e + 16);
    if (eocd >= 20 && rd32(e - 20) == 0x07064b50u) {  // zip64 locator
        const uint64_t z64 = rd64(e - 20 + 8);
        unsigned char z[56];
        if (z64 + 56 > fsize || !read_at(f, z64, 56, z) || rd32(z) != 0x06064b50u) {
            err = "bad zip64 record: " + path;
            return false;
        }
        n_entries = rd64(z + 32);
        cd_size = rd64(z + 40);
        cd_off = rd64(z + 48);
    }
    if (cd_off + cd_size > fsize) { err = "bad central directory: " + path; return false; }
    std::vector<unsigned char> cd((size_t)cd_size);
    if (!read_at(f, cd_off, (size_t)cd_size, cd.data())) { err = "read failed: " + path; return false; }
    uint64_t p = 0;
    for (uint64_t k = 0; k < n_entries; ++k) {
        if (p + 46 > cd_size || rd32(cd.data() + p) != 0x02014b50u) { err = "bad central directory: " + path; return false; }
        const unsigned char* c = cd.data() + p;
        const int method = rd16(c + 10);
        const uint32_t crc_expect = rd32(c + 16);
        uint64_t csize = rd32(c + 20), usize = rd32(c + 24);
        const int nlen = rd16(c + 28), xlen = rd16(c + 30), clen = rd16(c + 32);
        uint64_t loff = rd32(c + 42);
        if (p + 46 + (uint64_t)nlen + xlen > cd_size) { err = "bad central directory: " + path; return false; }
        std::string name(reinterpret_cast<const char*>(c + 46), nlen);
        // zip64 extra field: present values replace the 0xffffffff markers in order
        const unsigned char* x = c + 46 + nlen;
        for (int q = 0; q + 4 <= xlen;) {
            const int id = rd16(x + q), sz = rd16(x + q + 2);
            if (id == 0x0001) {
                int r = q + 4;
                if (usize == 0xffffffffu && r + 8 <= q + 4 + sz) { usize = rd64(x + r); r += 8; }
                if (csize == 0xffffffffu && r + 8 <= q + 4 + sz) { csize = rd64(x + r); r += 8; }
                if (loff == 0xffffffffu && r + 8 <= q + 4 + sz) { loff = rd64(x + r); r += 8; }
            }
            q += 4 + sz;
        }
        p += 46 + (uint64_t)nlen + xlen + clen;
        std::string key = name;
        if (key.size() > 4 && key.compare(key.size() - 4, 4, ".npy") == 0) key = key.substr(0, key.size() - 4);
        if (names) names->push_back(key);
        if (only && std::find(only->begin(), only->end(), key) == only->end()) continue;
        unsigned char lh[30];
        if (loff + 30 > fsize || !read_at(f, loff, 30, lh) || rd32(lh) != 0x04034b50u) {
            err = "bad local header: " + name;
            return false;
        }
        const uint64_t data = loff + 30 + rd16(lh + 26) + rd16(lh + 28);
        if (data + csize > fsize) { err = "truncated member: " + name; return false; }
        std::vector<char> raw((size_t)csize);
        if (!read_at(f, data, (size_t)csize, raw.data())) { err = "read failed: " + name; return false; }
        std::vector<char> inflated;
        const char* buf;
        size_t blen;
        if (method == 0) {
            buf = raw.data();
            blen = raw.size();
        } else if (method == 8) {
            if (!inflate_raw(reinterpret_cast<const unsigned char*>(raw.data()), raw.size(), inflated, (size_t)usize,
                             err)) {
                err += ": " + name;
                return false;
            }
            buf = inflated.data();
            blen = inflated.size();
        } else {
            err = "unsupported zip compression method in " + name;
            return false;
        }
        if (blen != usize) { err = "member size differs from its directory entry: " + name; return false; }
        {   // CRC-32 of the member's uncompressed bytes against its central-directory entry
            uLong crc = crc32(0L, Z_NULL, 0);
            for (size_t at = 0; at < blen;) {
                const size_t n = std::min<size_t>(blen - at, (size_t)1 << 30);
                crc = crc32(crc, reinterpret_cast<const Bytef*>(buf + at), (uInt)n);
                at += n;
            }
            if ((uint32_t)crc != crc_expect) { err = "CRC-32 mismatch (corrupt member): " + name; return false; }
        }
        NpyArray a;
        if (!npy_parse(buf, blen, a, err)) { err += " (" + name + ")"; return false; }
        out[key] = std::move(a);
    }
    return true;
}

}  // namespace dtb
