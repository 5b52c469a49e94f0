// Test driver for the block I/O of the processor executable (mdaio.cpp):
// prints what RowReader reads and does what RowWriter is asked, so that
// tests/test_mdaio_rows.py can check both against numpy without a GPU.
//
//   read <path> <as: f32|i16> <t0> <nt> <out.bin>   rows [t0, t0+nt) as raw bytes
//   info <path>                                      "M N dtype"
//   write <path> <dtype: f32|i16> <M> <N> <t0> <in.bin> [abort]
//                                                    one block at t0 from in.bin, then commit (or not)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mdaio.h"

static int fail(const std::string& e) {
    std::fprintf(stderr, "%s\n", e.c_str());
    return 1;
}

int main(int argc, char** argv) {
    if (argc < 3) return fail("usage");
    const std::string cmd = argv[1];
    std::string err;
    if (cmd == "info") {
        ms3io::RowReader r;
        if (!r.open(argv[2], err)) return fail(err);
        std::printf("%lld %lld %d\n", (long long)r.M(), (long long)r.N(), r.data_type());
        return 0;
    }
    if (cmd == "read" && argc == 7) {
        ms3io::RowReader r;
        if (!r.open(argv[2], err)) return fail(err);
        const int32_t as = std::string(argv[3]) == "i16" ? ms3io::kInt16 : ms3io::kFloat32;
        const int64_t t0 = std::atoll(argv[4]), nt = std::atoll(argv[5]);
        std::vector<unsigned char> buf((size_t)(nt * r.M()) * (as == ms3io::kInt16 ? 2 : 4) + 1);
        if (!r.read(t0, nt, as, buf.data(), err)) return fail(err);
        FILE* f = std::fopen(argv[6], "wb");
        if (!f) return fail("cannot write output");
        std::fwrite(buf.data(), 1, buf.size() - 1, f);
        std::fclose(f);
        return 0;
    }
    if (cmd == "write" && argc >= 8) {
        const int32_t dt = std::string(argv[3]) == "i16" ? ms3io::kInt16 : ms3io::kFloat32;
        const int64_t M = std::atoll(argv[4]), N = std::atoll(argv[5]), t0 = std::atoll(argv[6]);
        FILE* f = std::fopen(argv[7], "rb");
        if (!f) return fail("cannot read block");
        std::vector<unsigned char> buf;
        unsigned char tmp[65536];
        size_t k;
        while ((k = std::fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + k);
        std::fclose(f);
        const int64_t nt = (int64_t)buf.size() / (M * (dt == ms3io::kInt16 ? 2 : 4));
        ms3io::RowWriter w;
        if (!w.open(argv[2], dt, M, N, err)) return fail(err);
        if (!w.write(t0, nt, buf.data(), err)) return fail(err);
        if (argc == 9 && std::string(argv[8]) == "abort") return 0;  // destructor removes the .tmp file
        if (!w.commit(err)) return fail(err);
        return 0;
    }
    return fail("bad command");
}
