// Host driver for tests/test_regdft.py: runs the register DFTs of
// mountainsort_b200/csrc/fft_reg.cuh (RegDft, compile-time twiddle tables)
// on the CPU.  The header's functions are __host__ __device__, so this is
// the same source the bandpass kernels unroll.
//
//   regdft_driver dft N INV in.bin out.bin count   count N-point transforms (float2)
//   regdft_driver roots N out.bin                   the RootTable<N> values (re, im)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fft_reg.cuh"

using namespace ms3gpu;

template <int N, bool INV>
static void run_all(std::vector<float2>& v, long count) {
    for (long c = 0; c < count; c++) RegDft<N, INV>::run(v.data() + c * N);
}

template <int N>
static bool dispatch_inv(bool inv, std::vector<float2>& v, long count) {
    if (inv)
        run_all<N, true>(v, count);
    else
        run_all<N, false>(v, count);
    return true;
}

static bool dispatch(int n, bool inv, std::vector<float2>& v, long count) {
    switch (n) {
        case 2: return dispatch_inv<2>(inv, v, count);
        case 3: return dispatch_inv<3>(inv, v, count);
        case 4: return dispatch_inv<4>(inv, v, count);
        case 5: return dispatch_inv<5>(inv, v, count);
        case 8: return dispatch_inv<8>(inv, v, count);
        case 15: return dispatch_inv<15>(inv, v, count);
        case 16: return dispatch_inv<16>(inv, v, count);
        case 20: return dispatch_inv<20>(inv, v, count);
        case 25: return dispatch_inv<25>(inv, v, count);
        case 30: return dispatch_inv<30>(inv, v, count);
        default: return false;
    }
}

template <int N>
static void roots(std::vector<float>& out) {
    constexpr ct::RootTable<N> t = ct::RootTable<N>();
    for (int e = 0; e < N; e++) {
        out.push_back(t.re[e]);
        out.push_back(t.im[e]);
    }
}

static bool dispatch_roots(int n, std::vector<float>& out) {
    switch (n) {
        case 15: roots<15>(out); return true;
        case 16: roots<16>(out); return true;
        case 20: roots<20>(out); return true;
        case 25: roots<25>(out); return true;
        case 30: roots<30>(out); return true;
        default: return false;
    }
}

int main(int argc, char** argv) {
    if (argc >= 7 && !std::strcmp(argv[1], "dft")) {
        const int n = std::atoi(argv[2]);
        const bool inv = std::atoi(argv[3]) != 0;
        const long count = std::atol(argv[6]);
        std::vector<float2> v((size_t)n * count);
        FILE* f = std::fopen(argv[4], "rb");
        if (!f || std::fread(v.data(), sizeof(float2), v.size(), f) != v.size()) return 2;
        std::fclose(f);
        if (!dispatch(n, inv, v, count)) return 3;
        f = std::fopen(argv[5], "wb");
        if (!f || std::fwrite(v.data(), sizeof(float2), v.size(), f) != v.size()) return 2;
        std::fclose(f);
        return 0;
    }
    if (argc >= 4 && !std::strcmp(argv[1], "roots")) {
        std::vector<float> out;
        if (!dispatch_roots(std::atoi(argv[2]), out)) return 3;
        FILE* f = std::fopen(argv[3], "wb");
        if (!f || std::fwrite(out.data(), sizeof(float), out.size(), f) != out.size()) return 2;
        std::fclose(f);
        return 0;
    }
    std::fprintf(stderr, "usage: regdft_driver dft N INV in out count | roots N out\n");
    return 1;
}
