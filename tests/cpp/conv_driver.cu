// Host driver for tests/test_conversions.py: the float -> int16 and
// double -> int32 conversions of mountainsort_b200/csrc/common.cuh
// (__host__ __device__: the same source the output kernels use).
//
//   conv_driver f2i16 in.bin out.bin   float32 in, int16 out
//   conv_driver d2i32 in.bin out.bin   float64 in, int32 out
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"

template <class In, class Out, class F>
static int run(const char* in, const char* out, F f) {
    FILE* fi = std::fopen(in, "rb");
    if (!fi) return 2;
    std::fseek(fi, 0, SEEK_END);
    const long bytes = std::ftell(fi);
    std::fseek(fi, 0, SEEK_SET);
    std::vector<In> x((size_t)(bytes / (long)sizeof(In)));
    if (std::fread(x.data(), sizeof(In), x.size(), fi) != x.size()) return 2;
    std::fclose(fi);
    std::vector<Out> y(x.size());
    for (size_t i = 0; i < x.size(); i++) y[i] = f(x[i]);
    FILE* fo = std::fopen(out, "wb");
    if (!fo || std::fwrite(y.data(), sizeof(Out), y.size(), fo) != y.size()) return 2;
    std::fclose(fo);
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 4 && !std::strcmp(argv[1], "f2i16"))
        return run<float, int16_t>(argv[2], argv[3], [](float v) { return ms3gpu::x86_float_to_int16(v); });
    if (argc >= 4 && !std::strcmp(argv[1], "d2i32"))
        return run<double, int32_t>(argv[2], argv[3], [](double v) { return ms3gpu::x86_double_to_int32(v); });
    std::fprintf(stderr, "usage: conv_driver f2i16|d2i32 in out\n");
    return 1;
}
