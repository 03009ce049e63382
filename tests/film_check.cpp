// film_check.cpp - writes a film given as raw FP64 sums through the library's own .hdr writer
// (tr_film_io.cpp), so the CPU tests can compare its bytes with the RGBE encoding the GPU tests
// restate.  Usage: film_check <in.bin> <out name> W H T; in.bin = streak [H][W][T][3],
// steady [H][W][3], weight [H][W] as doubles.
#include "tr_film_io.h"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

int main(int argc, char** argv) {
    if (argc != 6) return 2;
    const uint32_t W = (uint32_t)std::strtoul(argv[3], nullptr, 10);
    const uint32_t H = (uint32_t)std::strtoul(argv[4], nullptr, 10);
    const uint32_t T = (uint32_t)std::strtoul(argv[5], nullptr, 10);
    const size_t np = (size_t)W * H, ns = np * T * 3, nd = np * 3;
    std::vector<double> buf(ns + nd + np);
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    const size_t got = std::fread(buf.data(), sizeof(double), buf.size(), f);
    std::fclose(f);
    if (got != buf.size()) return 4;
    std::string err;
    if (!trio::write_streak_film(argv[2], W, H, T, buf.data(), buf.data() + ns, buf.data() + ns + nd, &err)) {
        std::fprintf(stderr, "%s\n", err.c_str());
        return 5;
    }
    return 0;
}
