// Minimal .npy / .npz reader for the reference's block files
// (generation/make_block.py:473-479 writes them with numpy.savez).
#pragma once

#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace dtb {

struct NpyArray {
    std::string descr;            // numpy dtype string, e.g. "<f4", "|u1"
    bool fortran = false;
    std::vector<int64_t> shape;
    std::vector<char> data;       // raw little-endian bytes
    int64_t count() const
    {
        int64_t c = 1;
        for (int64_t s : shape) c *= s;
        return c;
    }
    int item_size() const;
};

// Parses one .npy buffer. Returns false and sets err on failure.
bool npy_parse(const char* buf, size_t len, NpyArray& out, std::string& err);

// Reads the members of a .npz (ZIP; stored or deflate; ZIP64 aware): all of
// them, or those named in `only` (names without ".npy").  `names` (nullable)
// receives every member name.
bool npz_read(const std::string& path, std::map<std::string, NpyArray>& out, std::string& err,
              const std::vector<std::string>* only = nullptr, std::vector<std::string>* names = nullptr);

}  // namespace dtb
