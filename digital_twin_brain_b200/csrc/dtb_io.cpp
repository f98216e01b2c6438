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

bool npz_read(const std::string& path, std::map<std::string, NpyArray>& out, std::string& err,
              const std::vector<std::string>* only, std::vector<std::string>* names)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) { err = "cannot open " + path; return false; }
    std::fseek(f, 0, SEEK_END);
    const long long fsize = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (fsize < 22) { std::fclose(f); err = "file too small for a zip archive: " + path; return false; }
    std::vector<unsigned char> file((size_t)fsize);
    if (std::fread(file.data(), 1, file.size(), f) != file.size()) { std::fclose(f); err = "read failed: " + path; return false; }
    std::fclose(f);
    const unsigned char* b = file.data();
    // end of central directory
    long long eocd = -1;
    for (long long i = fsize - 22; i >= 0 && i >= fsize - 22 - 65535; --i) {
        if (rd32(b + i) == 0x06054b50u) { eocd = i; break; }
    }
    if (eocd < 0) { err = "no end-of-central-directory record: " + path; return false; }
    uint64_t n_entries = rd16(b + eocd + 10);
    uint64_t cd_off = rd32(b + eocd + 16);
    if (eocd >= 20 && rd32(b + eocd - 20) == 0x07064b50u) {  // zip64 locator
        const uint64_t z64 = rd64(b + eocd - 20 + 8);
        if (z64 + 56 > (uint64_t)fsize || rd32(b + z64) != 0x06064b50u) { err = "bad zip64 record: " + path; return false; }
        n_entries = rd64(b + z64 + 32);
        cd_off = rd64(b + z64 + 48);
    }
    uint64_t p = cd_off;
    for (uint64_t e = 0; e < n_entries; ++e) {
        if (p + 46 > (uint64_t)fsize || rd32(b + p) != 0x02014b50u) { err = "bad central directory: " + path; return false; }
        const int method = rd16(b + p + 10);
        const uint32_t crc_expect = rd32(b + p + 16);
        uint64_t csize = rd32(b + p + 20), usize = rd32(b + p + 24);
        const int nlen = rd16(b + p + 28), xlen = rd16(b + p + 30), clen = rd16(b + p + 32);
        uint64_t loff = rd32(b + p + 42);
        std::string name(reinterpret_cast<const char*>(b + p + 46), nlen);
        // zip64 extra field: present values replace the 0xffffffff markers in order
        const unsigned char* x = b + p + 46 + nlen;
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
        {
            std::string key = name;
            if (key.size() > 4 && key.compare(key.size() - 4, 4, ".npy") == 0) key = key.substr(0, key.size() - 4);
            if (names) names->push_back(key);
            if (only && std::find(only->begin(), only->end(), key) == only->end()) continue;
        }
        if (loff + 30 > (uint64_t)fsize || rd32(b + loff) != 0x04034b50u) { err = "bad local header: " + name; return false; }
        const uint64_t data = loff + 30 + rd16(b + loff + 26) + rd16(b + loff + 28);
        if (data + csize > (uint64_t)fsize) { err = "truncated member: " + name; return false; }
        std::vector<char> raw;
        const char* buf;
        size_t blen;
        if (method == 0) {
            buf = reinterpret_cast<const char*>(b + data);
            blen = (size_t)csize;
        } else if (method == 8) {
            if (!inflate_raw(b + data, (size_t)csize, raw, (size_t)usize, err)) { err += ": " + name; return false; }
            buf = raw.data();
            blen = raw.size();
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
        std::string key = name;
        if (key.size() > 4 && key.compare(key.size() - 4, 4, ".npy") == 0) key = key.substr(0, key.size() - 4);
        NpyArray a;
        if (!npy_parse(buf, blen, a, err)) { err += " (" + name + ")"; return false; }
        out[key] = std::move(a);
    }
    return true;
}

}  // namespace dtb
