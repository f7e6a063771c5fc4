// Minimal .npy reader for the sorter's input directory.
//
// Replaces cnpy's loader as used by SorterHelpers.cpp:46-137 and
// OnlineSpikesV2.cu:550-608. Unlike cnpy (cnpy.cpp:62-73,181-184), it honours
// the header's fortran_order flag and returns the logical array in C order,
// converting the element type to the one the caller asks for.
#include "npy.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

namespace lss {

static bool parse_header(const std::string& hdr, NpyArray& a, std::string& err) {
    auto find_val = [&](const char* key) -> std::string {
        const size_t k = hdr.find(key);
        if (k == std::string::npos) return "";
        size_t c = hdr.find(':', k);
        if (c == std::string::npos) return "";
        return hdr.substr(c + 1);
    };
    std::string d = find_val("'descr'");
    const size_t q0 = d.find('\'');
    const size_t q1 = d.find('\'', q0 + 1);
    if (q0 == std::string::npos || q1 == std::string::npos) {
        err = "bad descr";
        return false;
    }
    a.descr = d.substr(q0 + 1, q1 - q0 - 1);
    std::string f = find_val("'fortran_order'");
    a.fortran = f.find("True") != std::string::npos && f.find("True") < f.find(',');
    std::string s = find_val("'shape'");
    const size_t p0 = s.find('('), p1 = s.find(')');
    if (p0 == std::string::npos || p1 == std::string::npos) {
        err = "bad shape";
        return false;
    }
    std::string inner = s.substr(p0 + 1, p1 - p0 - 1);
    a.shape.clear();
    std::stringstream ss(inner);
    std::string tok;
    while (std::getline(ss, tok, ',')) {
        size_t b = tok.find_first_not_of(" \t");
        if (b == std::string::npos) continue;
        a.shape.push_back(std::stoll(tok.substr(b)));
    }
    return true;
}

bool npy_load(const std::string& path, NpyArray& a, std::string& err) {
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        err = "cannot open " + path;
        return false;
    }
    char magic[6];
    in.read(magic, 6);
    if (!in || std::memcmp(magic, "\x93NUMPY", 6) != 0) {
        err = path + ": not a .npy file";
        return false;
    }
    unsigned char ver[2];
    in.read(reinterpret_cast<char*>(ver), 2);
    uint32_t hlen = 0;
    if (ver[0] == 1) {
        unsigned char b[2];
        in.read(reinterpret_cast<char*>(b), 2);
        hlen = b[0] | (b[1] << 8);
    } else {
        unsigned char b[4];
        in.read(reinterpret_cast<char*>(b), 4);
        hlen = b[0] | (b[1] << 8) | (b[2] << 16) | ((uint32_t)b[3] << 24);
    }
    std::string hdr(hlen, '\0');
    in.read(&hdr[0], hlen);
    if (!in || !parse_header(hdr, a, err)) {
        err = path + ": bad header " + err;
        return false;
    }
    if (a.descr.size() < 3 || (a.descr[0] != '<' && a.descr[0] != '|' && a.descr[0] != '=')) {
        err = path + ": unsupported dtype " + a.descr;
        return false;
    }
    a.kind = a.descr[1];
    a.itemsize = std::stoi(a.descr.substr(2));
    int64_t n = 1;
    for (auto d : a.shape) n *= d;
    a.raw.resize((size_t)n * a.itemsize);
    in.read(a.raw.data(), (std::streamsize)a.raw.size());
    if (!in) {
        err = path + ": truncated data";
        return false;
    }
    if (a.fortran && a.shape.size() > 1) {
        // logical C-order copy of a Fortran-ordered array
        std::vector<char> c(a.raw.size());
        const size_t nd = a.shape.size();
        std::vector<int64_t> idx(nd, 0);
        for (int64_t lin = 0; lin < n; ++lin) {
            int64_t fo = 0, stride = 1;
            for (size_t k = 0; k < nd; ++k) {
                fo += idx[k] * stride;
                stride *= a.shape[k];
            }
            std::memcpy(&c[(size_t)lin * a.itemsize], &a.raw[(size_t)fo * a.itemsize], a.itemsize);
            for (int k = (int)nd - 1; k >= 0; --k) {
                if (++idx[k] < a.shape[k]) break;
                idx[k] = 0;
            }
        }
        a.raw.swap(c);
        a.fortran = false;
    }
    return true;
}

template <typename T>
static bool convert(const NpyArray& a, std::vector<T>& out, std::string& err) {
    const size_t n = a.raw.size() / a.itemsize;
    out.resize(n);
    const char* p = a.raw.data();
    for (size_t i = 0; i < n; ++i) {
        const char* e = p + i * a.itemsize;
        double v;
        if (a.kind == 'f' && a.itemsize == 4) { float f; std::memcpy(&f, e, 4); v = f; }
        else if (a.kind == 'f' && a.itemsize == 8) { std::memcpy(&v, e, 8); }
        else if (a.kind == 'i' && a.itemsize == 8) { int64_t x; std::memcpy(&x, e, 8); out[i] = (T)x; continue; }
        else if (a.kind == 'i' && a.itemsize == 4) { int32_t x; std::memcpy(&x, e, 4); v = x; }
        else if (a.kind == 'i' && a.itemsize == 2) { int16_t x; std::memcpy(&x, e, 2); v = x; }
        else if (a.kind == 'u' && a.itemsize == 4) { uint32_t x; std::memcpy(&x, e, 4); v = x; }
        else { err = "unsupported dtype " + a.descr; return false; }
        out[i] = (T)v;
    }
    return true;
}

bool npy_as_f32(const NpyArray& a, std::vector<float>& out, std::string& err) { return convert(a, out, err); }
bool npy_as_i64(const NpyArray& a, std::vector<int64_t>& out, std::string& err) { return convert(a, out, err); }

}  // namespace lss
