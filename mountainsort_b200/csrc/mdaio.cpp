// .mda file I/O for the ms3gpu.mp processor executable (see mdaio.h).
#include "mdaio.h"

#include <sys/stat.h>

#include <cstdio>
#include <cstring>
#include <memory>

namespace ms3io {

namespace {
struct FileCloser {
    void operator()(FILE* f) const {
        if (f) std::fclose(f);
    }
};
using FilePtr = std::unique_ptr<FILE, FileCloser>;

template <class S, class D>
void convert(const S* src, D* dst, int64_t n) {
    for (int64_t i = 0; i < n; i++) dst[i] = (D)src[i];
}
}  // namespace

int bytes_per_entry(int32_t t) {
    switch (t) {
        case kUint8: return 1;
        case -1: return 8;
        case kFloat32: return 4;
        case kInt16: return 2;
        case kInt32: return 4;
        case kUint16: return 2;
        case kFloat64: return 8;
        case kUint32: return 4;
        default: return 0;
    }
}

static bool read_header_file(FILE* f, MdaHeader& h, std::string& err) {
    int32_t v[3];
    if (std::fread(v, 4, 3, f) != 3) { err = "truncated .mda header"; return false; }
    h.data_type = v[0];
    // mdaio.cpp:84-87 accepts codes -7..-1; -1 (complex) cannot be read as a timeseries
    if (h.data_type < -7 || h.data_type >= -1) { err = "unsupported .mda data type " + std::to_string(h.data_type); return false; }
    h.bytes_per_entry = bytes_per_entry(h.data_type);
    if (v[1] <= 0 || v[1] > 8) { err = "bad bytes per entry in .mda header"; return false; }
    int32_t nd = v[2];
    if (nd == 0 || nd > 50 || nd < -50) { err = "bad number of dimensions in .mda header"; return false; }
    h.uses64bitdims = nd < 0;
    if (nd < 0) nd = -nd;
    h.dims.assign((size_t)nd, 1);
    for (int i = 0; i < nd; i++) {
        if (h.uses64bitdims) {
            int64_t d;
            if (std::fread(&d, 8, 1, f) != 1) { err = "truncated .mda dims"; return false; }
            h.dims[(size_t)i] = d;
        } else {
            int32_t d;
            if (std::fread(&d, 4, 1, f) != 1) { err = "truncated .mda dims"; return false; }
            h.dims[(size_t)i] = d;
        }
        if (h.dims[(size_t)i] < 0) { err = "negative dimension in .mda header"; return false; }
    }
    h.header_size = 12 + (int64_t)nd * (h.uses64bitdims ? 8 : 4);
    return true;
}

bool read_header(const std::string& path, MdaHeader& h, std::string& err) {
    struct stat st;
    if (stat(path.c_str(), &st) == 0 && S_ISDIR(st.st_mode)) {
        err = "directory (concatenated) inputs are not supported: " + path;
        return false;
    }
    FilePtr f(std::fopen(path.c_str(), "rb"));
    if (!f) { err = "cannot open " + path; return false; }
    return read_header_file(f.get(), h, err);
}

bool read_timeseries_f32(const std::string& path, int64_t& M, int64_t& N, std::vector<float>& data,
                         std::string& err) {
    MdaHeader h;
    if (!read_header(path, h, err)) return false;
    FilePtr f(std::fopen(path.c_str(), "rb"));
    if (!f) { err = "cannot open " + path; return false; }
    std::fseek(f.get(), (long)h.header_size, SEEK_SET);
    M = h.dims[0];
    N = h.dims.size() > 1 ? h.dims[1] : 1;
    const int64_t n = M * N;
    data.resize((size_t)n);
    const int bpe = h.bytes_per_entry;
    if (h.data_type == kFloat32) {
        if ((int64_t)std::fread(data.data(), 4, (size_t)n, f.get()) != n) { err = "short read from " + path; return false; }
        return true;
    }
    const int64_t block = 1 << 20;
    std::vector<unsigned char> buf((size_t)(block * bpe));
    for (int64_t i = 0; i < n; i += block) {
        const int64_t m = std::min(block, n - i);
        if ((int64_t)std::fread(buf.data(), (size_t)bpe, (size_t)m, f.get()) != m) { err = "short read from " + path; return false; }
        float* dst = data.data() + i;
        switch (h.data_type) {
            case kUint8: convert(reinterpret_cast<const uint8_t*>(buf.data()), dst, m); break;
            case kInt16: convert(reinterpret_cast<const int16_t*>(buf.data()), dst, m); break;
            case kInt32: convert(reinterpret_cast<const int32_t*>(buf.data()), dst, m); break;
            case kUint16: convert(reinterpret_cast<const uint16_t*>(buf.data()), dst, m); break;
            case kFloat64: convert(reinterpret_cast<const double*>(buf.data()), dst, m); break;
            default: err = "unsupported data type"; return false;
        }
    }
    return true;
}

bool write_timeseries(const std::string& path, int32_t data_type, int64_t M, int64_t N, const void* data,
                      std::string& err) {
    const std::string tmp = path + ".tmp";
    std::remove(path.c_str());
    FilePtr f(std::fopen(tmp.c_str(), "wb"));
    if (!f) { err = "cannot open " + tmp + " for writing"; return false; }
    const bool use64 = (M > 2e9) || (N > 2e9);
    const int32_t hdr[3] = {data_type, (int32_t)bytes_per_entry(data_type), use64 ? -2 : 2};
    bool ok = std::fwrite(hdr, 4, 3, f.get()) == 3;
    if (use64) {
        const int64_t d[2] = {M, N};
        ok = ok && std::fwrite(d, 8, 2, f.get()) == 2;
    } else {
        const int32_t d[2] = {(int32_t)M, (int32_t)N};
        ok = ok && std::fwrite(d, 4, 2, f.get()) == 2;
    }
    const size_t n = (size_t)(M * N);
    if (n) ok = ok && std::fwrite(data, (size_t)bytes_per_entry(data_type), n, f.get()) == n;
    ok = ok && std::fflush(f.get()) == 0;
    FILE* raw = f.release();
    ok = (std::fclose(raw) == 0) && ok;
    if (!ok) {
        std::remove(tmp.c_str());
        err = "write failed for " + tmp;
        return false;
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        err = "cannot rename " + tmp + " to " + path;
        return false;
    }
    return true;
}

bool copy_file(const std::string& src, const std::string& dst, std::string& err) {
    struct stat st;
    if (stat(dst.c_str(), &st) == 0) { err = "destination exists: " + dst; return false; }
    FilePtr in(std::fopen(src.c_str(), "rb"));
    if (!in) { err = "cannot open " + src; return false; }
    FilePtr out(std::fopen(dst.c_str(), "wb"));
    if (!out) { err = "cannot open " + dst; return false; }
    std::vector<char> buf(1 << 22);
    size_t n;
    while ((n = std::fread(buf.data(), 1, buf.size(), in.get())) > 0)
        if (std::fwrite(buf.data(), 1, n, out.get()) != n) { err = "write failed for " + dst; return false; }
    return true;
}

}  // namespace ms3io

namespace ms3io {

namespace {
// All entries of an array converted to D (std::copy semantics, like the
// reference's mdaReadData, mdaio.cpp:205-230).
template <class D>
bool read_entries(const std::string& path, std::vector<int64_t>& dims, std::vector<D>& data, std::string& err) {
    MdaHeader h;
    if (!read_header(path, h, err)) return false;
    FilePtr f(std::fopen(path.c_str(), "rb"));
    if (!f) { err = "cannot open " + path; return false; }
    std::fseek(f.get(), (long)h.header_size, SEEK_SET);
    dims = h.dims;
    int64_t n = 1;
    for (int64_t d : dims) n *= d;
    data.resize((size_t)n);
    const int64_t block = 1 << 20;
    const int bpe = h.bytes_per_entry;
    std::vector<unsigned char> buf((size_t)(block * bpe));
    for (int64_t i = 0; i < n; i += block) {
        const int64_t m = std::min(block, n - i);
        if ((int64_t)std::fread(buf.data(), (size_t)bpe, (size_t)m, f.get()) != m) { err = "short read from " + path; return false; }
        D* dst = data.data() + i;
        switch (h.data_type) {
            case kUint8: convert(reinterpret_cast<const uint8_t*>(buf.data()), dst, m); break;
            case kFloat32: convert(reinterpret_cast<const float*>(buf.data()), dst, m); break;
            case kInt16: convert(reinterpret_cast<const int16_t*>(buf.data()), dst, m); break;
            case kInt32: convert(reinterpret_cast<const int32_t*>(buf.data()), dst, m); break;
            case kUint16: convert(reinterpret_cast<const uint16_t*>(buf.data()), dst, m); break;
            case kFloat64: convert(reinterpret_cast<const double*>(buf.data()), dst, m); break;
            case kUint32: convert(reinterpret_cast<const uint32_t*>(buf.data()), dst, m); break;
            default: err = "unsupported data type"; return false;
        }
    }
    return true;
}
}  // namespace

bool read_array_f32(const std::string& path, std::vector<int64_t>& dims, std::vector<float>& data,
                    std::string& err) {
    return read_entries(path, dims, data, err);
}

bool read_array_f64(const std::string& path, std::vector<int64_t>& dims, std::vector<double>& data,
                    std::string& err) {
    return read_entries(path, dims, data, err);
}

bool write_array(const std::string& path, int32_t data_type, const std::vector<int64_t>& dims, const void* data,
                 std::string& err) {
    const std::string tmp = path + ".tmp";
    std::remove(path.c_str());
    FilePtr f(std::fopen(tmp.c_str(), "wb"));
    if (!f) { err = "cannot open " + tmp + " for writing"; return false; }
    bool use64 = false;
    int64_t n = 1;
    for (int64_t d : dims) {
        use64 = use64 || d > 2e9;
        n *= d;
    }
    const int32_t nd = (int32_t)dims.size();
    const int32_t hdr[3] = {data_type, (int32_t)bytes_per_entry(data_type), use64 ? -nd : nd};
    bool ok = std::fwrite(hdr, 4, 3, f.get()) == 3;
    for (int64_t d : dims) {
        if (use64) {
            ok = ok && std::fwrite(&d, 8, 1, f.get()) == 1;
        } else {
            const int32_t d32 = (int32_t)d;
            ok = ok && std::fwrite(&d32, 4, 1, f.get()) == 1;
        }
    }
    if (n) ok = ok && std::fwrite(data, (size_t)bytes_per_entry(data_type), (size_t)n, f.get()) == (size_t)n;
    ok = ok && std::fflush(f.get()) == 0;
    FILE* raw = f.release();
    ok = (std::fclose(raw) == 0) && ok;
    if (!ok) {
        std::remove(tmp.c_str());
        err = "write failed for " + tmp;
        return false;
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        err = "cannot rename " + tmp + " to " + path;
        return false;
    }
    return true;
}

}  // namespace ms3io
