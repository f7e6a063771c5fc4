// .npy reading for the sorter's input directory (see npy.cpp).
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace lss {

struct NpyArray {
    std::string descr;
    char kind = 0;        // 'f', 'i', 'u'
    int itemsize = 0;
    bool fortran = false; // always false after npy_load (converted to C order)
    std::vector<int64_t> shape;
    std::vector<char> raw;
    int64_t numel() const {
        int64_t n = 1;
        for (auto d : shape) n *= d;
        return n;
    }
};

bool npy_load(const std::string& path, NpyArray& a, std::string& err);
bool npy_as_f32(const NpyArray& a, std::vector<float>& out, std::string& err);
bool npy_as_i64(const NpyArray& a, std::vector<int64_t>& out, std::string& err);

}  // namespace lss
