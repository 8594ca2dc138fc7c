// Image files for the task queue's read-in and write-out callbacks: the
// reference's readInFuncs / writeOutFuncs (src/imresh/io/readInFuncs/readInFuncs.hpp:57-84,
// src/imresh/io/writeOutFuncs/writeOutFuncs.hpp:52-106) for formats that need
// no third-party library -- NumPy .npy (float32 or float64, 2-D, C order),
// whitespace-separated text (one image row per line) and headerless float32
// (width contiguous).  PNG, TIFF and HDF5 need pngwriter, libtiff and
// libSplash, which are not part of this build.
//
// Buffers handed out by the readers come from new[], so justFree and the
// *AndFree writers release them, as in the reference.  Failures print to
// stderr and return an error (the reference exits the process).
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "imresh_b200.h"
#include "imresh/io/readInFuncs/readInFuncs.hpp"
#include "imresh/io/writeOutFuncs/writeOutFuncs.hpp"

namespace {

int fail(const char *what, const char *path)
{
    fprintf(stderr, "imresh_b200 io: %s: %s\n", what, path ? path : "(null)");
    return IMR_ERR_INVALID_VALUE;
}

bool little_endian()
{
    const uint16_t one = 1;
    unsigned char c;
    memcpy(&c, &one, 1);
    return c == 1;
}

// value of `key` in a .npy header dictionary (text after "'key':")
std::string npy_field(const std::string &h, const char *key)
{
    const std::string k = std::string("'") + key + "'";
    size_t p = h.find(k);
    if (p == std::string::npos) return "";
    p = h.find(':', p + k.size());
    if (p == std::string::npos) return "";
    ++p;
    while (p < h.size() && isspace((unsigned char)h[p])) ++p;
    size_t e = p;
    if (p < h.size() && h[p] == '(') {
        e = h.find(')', p);
        return e == std::string::npos ? "" : h.substr(p, e - p + 1);
    }
    while (e < h.size() && h[e] != ',' && h[e] != '}') ++e;
    return h.substr(p, e - p);
}

}  // namespace

extern "C" {

void imr_free_image(float *data) { delete[] data; }

int imr_write_npy(const char *path, const float *data, unsigned W, unsigned H)
{
    if (!path || !data || W == 0 || H == 0) return fail("invalid arguments to the .npy writer", path);
    if (!little_endian()) return fail("the .npy writer needs a little-endian host", path);
    std::string dict = "{'descr': '<f4', 'fortran_order': False, 'shape': (" + std::to_string(H) + ", " +
                       std::to_string(W) + "), }";
    size_t total = 10 + dict.size() + 1;   // magic, version, length, dict, '\n'
    dict.append((64 - total % 64) % 64, ' ');
    dict.push_back('\n');
    FILE *f = fopen(path, "wb");
    if (!f) return fail("cannot open for writing", path);
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    const uint16_t hl = (uint16_t)dict.size();
    bool ok = fwrite(magic, 1, 8, f) == 8 && fwrite(&hl, 2, 1, f) == 1 &&
              fwrite(dict.data(), 1, dict.size(), f) == dict.size() &&
              fwrite(data, sizeof(float), (size_t)W * H, f) == (size_t)W * H;
    ok = (fclose(f) == 0) && ok;
    return ok ? IMR_SUCCESS : fail("write failed", path);
}

int imr_read_npy(const char *path, float **data, unsigned *W, unsigned *H)
{
    if (!path || !data || !W || !H) return fail("invalid arguments to the .npy reader", path);
    *data = nullptr;
    *W = *H = 0;
    if (!little_endian()) return fail("the .npy reader needs a little-endian host", path);
    FILE *f = fopen(path, "rb");
    if (!f) return fail("cannot open", path);
    unsigned char pre[10];
    std::string hdr;
    bool ok = fread(pre, 1, 10, f) == 10 && memcmp(pre, "\x93NUMPY", 6) == 0;
    size_t hl = 0;
    if (ok && pre[6] == 1) {
        hl = (size_t)pre[8] | ((size_t)pre[9] << 8);
    } else if (ok && (pre[6] == 2 || pre[6] == 3)) {
        unsigned char x[2];
        ok = fread(x, 1, 2, f) == 2;
        hl = (size_t)pre[8] | ((size_t)pre[9] << 8) | ((size_t)x[0] << 16) | ((size_t)x[1] << 24);
    } else {
        ok = false;
    }
    if (ok) {
        hdr.resize(hl);
        ok = fread(&hdr[0], 1, hl, f) == hl;
    }
    if (!ok) {
        fclose(f);
        return fail("not a .npy file", path);
    }
    const std::string descr = npy_field(hdr, "descr"), order = npy_field(hdr, "fortran_order"),
                      shape = npy_field(hdr, "shape");
    const bool f4 = descr.find("<f4") != std::string::npos, f8 = descr.find("<f8") != std::string::npos;
    std::vector<unsigned long> dims;
    for (size_t p = 0; p < shape.size();) {
        if (isdigit((unsigned char)shape[p])) {
            size_t e = p;
            while (e < shape.size() && isdigit((unsigned char)shape[e])) ++e;
            dims.push_back(std::stoul(shape.substr(p, e - p)));
            p = e;
        } else {
            ++p;
        }
    }
    if ((!f4 && !f8) || order.find("False") == std::string::npos || dims.empty() || dims.size() > 2) {
        fclose(f);
        return fail("unsupported .npy layout (need 1-D or 2-D little-endian float32/float64, C order)", path);
    }
    const unsigned long h = dims.size() == 2 ? dims[0] : 1, w = dims.back();
    const size_t n = (size_t)w * h;
    if (n == 0 || w > 0xffffffffUL || h > 0xffffffffUL) {
        fclose(f);
        return fail("empty or oversized .npy array", path);
    }
    float *out = new float[n];
    if (f4) {
        ok = fread(out, sizeof(float), n, f) == n;
    } else {
        std::vector<double> tmp(n);
        ok = fread(tmp.data(), sizeof(double), n, f) == n;
        for (size_t i = 0; ok && i < n; ++i) out[i] = (float)tmp[i];
    }
    fclose(f);
    if (!ok) {
        delete[] out;
        return fail("truncated .npy data", path);
    }
    *data = out;
    *W = (unsigned)w;
    *H = (unsigned)h;
    return IMR_SUCCESS;
}

int imr_write_txt(const char *path, const float *data, unsigned W, unsigned H)
{
    if (!path || !data || W == 0 || H == 0) return fail("invalid arguments to the text writer", path);
    FILE *f = fopen(path, "w");
    if (!f) return fail("cannot open for writing", path);
    bool ok = true;
    for (unsigned y = 0; y < H && ok; ++y)
        for (unsigned x = 0; x < W && ok; ++x)
            ok = fprintf(f, x + 1 < W ? "%.9g " : "%.9g\n", (double)data[(size_t)y * W + x]) > 0;
    ok = (fclose(f) == 0) && ok;
    return ok ? IMR_SUCCESS : fail("write failed", path);
}

int imr_read_txt(const char *path, float **data, unsigned *W, unsigned *H)
{
    if (!path || !data || !W || !H) return fail("invalid arguments to the text reader", path);
    *data = nullptr;
    *W = *H = 0;
    std::ifstream in(path);
    if (!in.is_open()) return fail("cannot open", path);
    std::vector<float> vals;
    size_t w = 0, h = 0;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        size_t n = 0;
        std::string tok;
        while (ls >> tok) {
            char *end = nullptr;
            const float v = strtof(tok.c_str(), &end);
            if (end == tok.c_str() || *end != '\0') return fail("not a number in the text image", path);
            vals.push_back(v);
            ++n;
        }
        if (n == 0) continue;   // blank line
        if (w == 0) w = n;
        if (n != w) return fail("rows of different length in the text image", path);
        ++h;
    }
    if (vals.empty()) return fail("empty text image", path);
    float *out = new float[vals.size()];
    memcpy(out, vals.data(), vals.size() * sizeof(float));
    *data = out;
    *W = (unsigned)w;
    *H = (unsigned)h;
    return IMR_SUCCESS;
}

int imr_write_raw(const char *path, const float *data, unsigned W, unsigned H)
{
    if (!path || !data || W == 0 || H == 0) return fail("invalid arguments to the raw writer", path);
    FILE *f = fopen(path, "wb");
    if (!f) return fail("cannot open for writing", path);
    bool ok = fwrite(data, sizeof(float), (size_t)W * H, f) == (size_t)W * H;
    ok = (fclose(f) == 0) && ok;
    return ok ? IMR_SUCCESS : fail("write failed", path);
}

}  // extern "C"

namespace imresh
{
namespace io
{
namespace readInFuncs
{
    // Whitespace-separated numbers, one image row per line; xDim = values per
    // row (the reference counts them the same way, readInFuncs.cpp:55-70).
    FloatImage readTxt(std::string const filename)
    {
        float *d = nullptr;
        unsigned w = 0, h = 0;
        imr_read_txt(filename.c_str(), &d, &w, &h);
        return std::make_pair(d, std::make_pair(w, h));
    }
    FloatImage readNpy(std::string const filename)
    {
        float *d = nullptr;
        unsigned w = 0, h = 0;
        imr_read_npy(filename.c_str(), &d, &w, &h);
        return std::make_pair(d, std::make_pair(w, h));
    }
} // namespace readInFuncs

namespace writeOutFuncs
{
    void writeOutNpy(float *mem, unsigned int const w, unsigned int const h, std::string const fileName)
    {
        imr_write_npy(fileName.c_str(), mem, w, h);
    }
    void writeOutAndFreeNpy(float *mem, unsigned int const w, unsigned int const h, std::string const fileName)
    {
        writeOutNpy(mem, w, h, fileName);
        delete[] mem;
    }
    void writeOutTxt(float *mem, unsigned int const w, unsigned int const h, std::string const fileName)
    {
        imr_write_txt(fileName.c_str(), mem, w, h);
    }
    void writeOutAndFreeTxt(float *mem, unsigned int const w, unsigned int const h, std::string const fileName)
    {
        writeOutTxt(mem, w, h, fileName);
        delete[] mem;
    }
    void writeOutRaw(float *mem, unsigned int const w, unsigned int const h, std::string const fileName)
    {
        imr_write_raw(fileName.c_str(), mem, w, h);
    }
    void writeOutAndFreeRaw(float *mem, unsigned int const w, unsigned int const h, std::string const fileName)
    {
        writeOutRaw(mem, w, h, fileName);
        delete[] mem;
    }
} // namespace writeOutFuncs
} // namespace io
} // namespace imresh
