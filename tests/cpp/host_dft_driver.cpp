// Host driver for tests/test_host_dft.py: the FP64 transforms of
// mountainsort_b200/csrc/host_dft.h (the bandpass plan's table transforms:
// mixed radix, Bluestein for lengths with a prime factor above 64).
//
//   host_dft_driver dft S in.bin out.bin   complex128 in, its DFT with sign S out
//   host_dft_driver smooth N               prints next_smooth5(N)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "host_dft.h"

using ms3gpu::hostdft::cd;

int main(int argc, char** argv) {
    if (argc >= 5 && !std::strcmp(argv[1], "dft")) {
        const int s = std::atoi(argv[2]);
        FILE* f = std::fopen(argv[3], "rb");
        if (!f) return 2;
        std::fseek(f, 0, SEEK_END);
        const long bytes = std::ftell(f);
        std::fseek(f, 0, SEEK_SET);
        std::vector<cd> x((size_t)(bytes / (long)sizeof(cd)));
        if (std::fread(x.data(), sizeof(cd), x.size(), f) != x.size()) return 2;
        std::fclose(f);
        const std::vector<cd> y = ms3gpu::hostdft::dft(x, s);
        f = std::fopen(argv[4], "wb");
        if (!f || std::fwrite(y.data(), sizeof(cd), y.size(), f) != y.size()) return 2;
        std::fclose(f);
        return 0;
    }
    if (argc >= 3 && !std::strcmp(argv[1], "smooth")) {
        std::printf("%lld\n", (long long)ms3gpu::hostdft::next_smooth5(std::atoll(argv[2])));
        return 0;
    }
    std::fprintf(stderr, "usage: host_dft_driver dft S in out | smooth N\n");
    return 1;
}
