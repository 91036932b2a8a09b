// dropin_main.cpp -- a C++ caller of the drop-in entry points, written the
// way code that used the reference library calls it (2D/LibThinning2D.h,
// 3D/LibThinning3D.h, 2D/CenterlineExtraction.h, 3D/CenterlineExctraction.h):
// host arrays in, new[] outputs the caller delete[]s.  tests/test_dropin_cpp.py
// compiles it with g++ against include/ and libbgt.so and compares what it
// writes with the oracle.
//
//   dropin_main thin2d_u8  in.raw w h out.raw
//   dropin_main thin3d_f32 in.raw w h d out.raw        (uint8 in, converted to float)
//   dropin_main cl2d_u8    in.raw w h ml sp out_prefix (writes .x .y .idx)
//   dropin_main cl3d_u8    in.raw w h d ml sp out_prefix (writes .x .y .z .idx)
//   dropin_main bad_sizes                              (prints the results of invalid calls)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "CenterlineExctraction.h"
#include "CenterlineExtraction.h"
#include "LibThinning2D.h"
#include "LibThinning3D.h"

static std::vector<unsigned char> read_raw(const char *path, size_t n)
{
    std::vector<unsigned char> v(n);
    FILE *f = fopen(path, "rb");
    if (!f || fread(v.data(), 1, n, f) != n) {
        fprintf(stderr, "cannot read %s\n", path);
        exit(2);
    }
    fclose(f);
    return v;
}

template <typename T>
static void write_raw(const std::string &path, const T *p, size_t n)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f || (n && fwrite(p, sizeof(T), n, f) != n)) {
        fprintf(stderr, "cannot write %s\n", path.c_str());
        exit(2);
    }
    fclose(f);
}

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    const std::string mode = argv[1];
    if (mode == "thin2d_u8" && argc == 6) {
        const int w = atoi(argv[3]), h = atoi(argv[4]);
        std::vector<unsigned char> in = read_raw(argv[2], (size_t)w * h), out((size_t)w * h, 9);
        Thinning2D<unsigned char>(w, h, in.data(), out.data());
        write_raw(argv[5], out.data(), out.size());
        return 0;
    }
    if (mode == "thin3d_f32" && argc == 7) {
        const int w = atoi(argv[3]), h = atoi(argv[4]), d = atoi(argv[5]);
        const size_t n = (size_t)w * h * d;
        std::vector<unsigned char> raw = read_raw(argv[2], n);
        std::vector<float> in(raw.begin(), raw.end()), out(n, 9.0f);
        Thinning3D<float>(w, h, d, in.data(), out.data());
        std::vector<unsigned char> o8(n);
        for (size_t i = 0; i < n; i++) o8[i] = out[i] != 0.0f;
        write_raw(argv[6], o8.data(), n);
        return 0;
    }
    if (mode == "cl2d_u8" && argc == 8) {
        const int w = atoi(argv[3]), h = atoi(argv[4]), ml = atoi(argv[5]), sp = atoi(argv[6]);
        std::vector<unsigned char> in = read_raw(argv[2], (size_t)w * h);
        float *x = nullptr, *y = nullptr;
        unsigned int *idx = nullptr;
        const unsigned int n = CenterlineExtraction<unsigned char>(in.data(), w, h, ml, sp, &x, &y, &idx);
        const std::string pre = argv[7];
        write_raw(pre + ".x", x, idx[n]);
        write_raw(pre + ".y", y, idx[n]);
        write_raw(pre + ".idx", idx, (size_t)n + 1);
        delete[] x;
        delete[] y;
        delete[] idx;
        return 0;
    }
    if (mode == "cl3d_u8" && argc == 9) {
        const int w = atoi(argv[3]), h = atoi(argv[4]), d = atoi(argv[5]), ml = atoi(argv[6]), sp = atoi(argv[7]);
        std::vector<unsigned char> in = read_raw(argv[2], (size_t)w * h * d);
        float *x = nullptr, *y = nullptr, *z = nullptr;
        unsigned int *idx = nullptr;
        const unsigned int n = CenterlineExtraction<unsigned char>(in.data(), w, h, d, ml, sp, &x, &y, &z, &idx);
        const std::string pre = argv[8];
        write_raw(pre + ".x", x, idx[n]);
        write_raw(pre + ".y", y, idx[n]);
        write_raw(pre + ".z", z, idx[n]);
        write_raw(pre + ".idx", idx, (size_t)n + 1);
        delete[] x;
        delete[] y;
        delete[] z;
        delete[] idx;
        return 0;
    }
    if (mode == "bad_sizes") {
        unsigned char px[4] = {1, 1, 1, 1}, out[4] = {9, 9, 9, 9};
        float *x = nullptr, *y = nullptr, *z = nullptr;
        unsigned int *idx = nullptr;
        const unsigned int n2 = CenterlineExtraction<unsigned char>(px, -5, 2, 10, 3, &x, &y, &idx);
        printf("cl2d %u %u\n", n2, idx ? idx[0] : 99u);
        delete[] x;
        delete[] y;
        delete[] idx;
        const unsigned int n3 = CenterlineExtraction<unsigned char>(px, 2, 2, 0, 10, 3, &x, &y, &z, &idx);
        printf("cl3d %u %u\n", n3, idx ? idx[0] : 99u);
        delete[] x;
        delete[] y;
        delete[] z;
        delete[] idx;
        // wider than the 32767-pixel limit: the call fails and zero-fills its output
        std::vector<unsigned char> wide_in(40000, 1), wide_out(40000, 9);
        Thinning2D<unsigned char>(40000, 1, wide_in.data(), wide_out.data());
        size_t nonzero = 0;
        for (unsigned char v : wide_out) nonzero += v != 0;
        printf("thin2d %zu\n", nonzero);
        (void)out;
        return 0;
    }
    fprintf(stderr, "bad arguments\n");
    return 2;
}
