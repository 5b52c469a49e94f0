// .mda file I/O for the ms3gpu.mp processor executable (see mdaio.h).
#include "mdaio.h"

#include <dirent.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>

#include <cstdio>
#include <cstring>
#include <memory>
#include <thread>

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

bool is_directory(const std::string& path) {
    struct stat st;
    return stat(path.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

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
    if (is_directory(path)) {
        err = "expected an .mda file, got a directory: " + path;
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

namespace ms3io {

// DiskReadMda32Private::find_all_mda_files_in_directory (recursive), mda/
// diskreadmda32.cpp:896-913: the directory's files ending in ".mda", sorted
// by name (QDir::Name: case-sensitive code-point order), then for every
// subdirectory (sorted) the files of `dir_path + "/dirname"` -- the
// reference appends the literal text "dirname", not the subdirectory's
// name, and that is kept.
void concat_directory_files(const std::string& dir, std::vector<std::string>& out) {
    std::vector<std::string> files, dirs;
    if (DIR* d = opendir(dir.c_str())) {
        while (dirent* e = readdir(d)) {
            const std::string n = e->d_name;
            if (n == "." || n == "..") continue;
            struct stat st;
            if (stat((dir + "/" + n).c_str(), &st) != 0) continue;
            if (S_ISDIR(st.st_mode))
                dirs.push_back(n);
            else if (S_ISREG(st.st_mode) && n.size() >= 4 && n.compare(n.size() - 4, 4, ".mda") == 0)
                files.push_back(n);
        }
        closedir(d);
    }
    std::sort(files.begin(), files.end());
    std::sort(dirs.begin(), dirs.end());
    for (const std::string& n : files) out.push_back(dir + "/" + n);
    for (size_t i = 0; i < dirs.size(); i++) concat_directory_files(dir + "/dirname", out);
}

bool input_files(const std::string& path, std::vector<std::string>& files, std::string& err) {
    files.clear();
    if (!is_directory(path)) {
        files.push_back(path);
        return true;
    }
    concat_directory_files(path, files);
    if (files.empty()) {
        err = "no .mda files in directory " + path;
        return false;
    }
    return true;
}

bool read_dims_any(const std::string& path, int64_t& M, int64_t& N, int32_t& data_type, std::string& err) {
    std::vector<std::string> files;
    if (!input_files(path, files, err)) return false;
    M = -1;
    N = 0;
    for (const std::string& f : files) {
        MdaHeader h;
        if (!read_header(f, h, err)) return false;
        const int64_t m = h.dims[0], n = h.dims.size() > 1 ? h.dims[1] : 1;
        if (M >= 0 && m != M) {
            err = "the files of " + path + " differ in channel count";
            return false;
        }
        data_type = (M < 0 || data_type == h.data_type) ? h.data_type : 0;  // 0: mixed types
        M = m;
        N += n;
    }
    return true;
}

bool read_timeseries_any_f32(const std::string& path, int64_t& M, int64_t& N, std::vector<float>& data,
                             std::string& err) {
    std::vector<std::string> files;
    if (!input_files(path, files, err)) return false;
    if (files.size() == 1) return read_timeseries_f32(files[0], M, N, data, err);
    M = -1;
    N = 0;
    data.clear();
    std::vector<float> part;
    for (const std::string& f : files) {
        int64_t m = 0, n = 0;
        if (!read_timeseries_f32(f, m, n, part, err)) return false;
        if (M >= 0 && m != M) {
            err = "the files of " + path + " differ in channel count";
            return false;
        }
        M = m;
        N += n;
        data.insert(data.end(), part.begin(), part.end());  // column-major M x n: append in time
    }
    return true;
}

bool read_timeseries_i16(const std::string& path, int64_t& M, int64_t& N, std::vector<int16_t>& data,
                         std::string& err) {
    MdaHeader h;
    if (!read_header(path, h, err)) return false;
    if (h.data_type != kInt16) {
        err = path + " is not int16";
        return false;
    }
    FilePtr f(std::fopen(path.c_str(), "rb"));
    if (!f) { err = "cannot open " + path; return false; }
    std::fseek(f.get(), (long)h.header_size, SEEK_SET);
    M = h.dims[0];
    N = h.dims.size() > 1 ? h.dims[1] : 1;
    data.resize((size_t)(M * N));
    if ((int64_t)std::fread(data.data(), 2, (size_t)(M * N), f.get()) != M * N) { err = "short read from " + path; return false; }
    return true;
}

}  // namespace ms3io

namespace ms3io {

namespace {
// pread / pwrite of the whole range (they may move fewer bytes per call)
bool pread_all(int fd, void* dst, size_t n, int64_t off) {
    char* p = static_cast<char*>(dst);
    while (n > 0) {
        const ssize_t r = ::pread(fd, p, n, (off_t)off);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return false;
        p += r;
        n -= (size_t)r;
        off += r;
    }
    return true;
}

bool pwrite_all(int fd, const void* src, size_t n, int64_t off) {
    const char* p = static_cast<const char*>(src);
    while (n > 0) {
        const ssize_t r = ::pwrite(fd, p, n, (off_t)off);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return false;
        p += r;
        n -= (size_t)r;
        off += r;
    }
    return true;
}

// A large block is moved by several threads, each with its own part: reads
// from the page cache scale with threads (one thread copies about 5 GB/s),
// buffered writes up to about two to four.
template <class F>
bool in_parts(size_t n, int max_threads, F&& part) {
    const size_t kMinPart = size_t(32) << 20;
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int T = (int)std::min<size_t>((size_t)std::min(max_threads, hw), std::max<size_t>(1, n / kMinPart));
    if (T <= 1) return part(0, n);
    const size_t per = ((n + T - 1) / T + 4095) & ~size_t(4095);
    std::vector<std::thread> th;
    std::vector<char> ok((size_t)T, 1);
    for (int i = 0; i < T; i++) {
        const size_t a = std::min(n, (size_t)i * per), b = std::min(n, a + per);
        if (a < b) th.emplace_back([&, i, a, b] { ok[(size_t)i] = part(a, b) ? 1 : 0; });
    }
    for (std::thread& t : th) t.join();
    return std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; });
}
}  // namespace

RowReader::~RowReader() {
    for (Seg& g : segs_)
        if (g.fd >= 0) ::close(g.fd);
}

bool RowReader::open(const std::string& path, std::string& err) {
    std::vector<std::string> files;
    if (!input_files(path, files, err)) return false;
    M_ = -1;
    N_ = 0;
    for (const std::string& f : files) {
        MdaHeader h;
        if (!read_header(f, h, err)) return false;
        const int64_t m = h.dims[0], n = h.dims.size() > 1 ? h.dims[1] : 1;
        if (M_ >= 0 && m != M_) {
            err = "the files of " + path + " differ in channel count";
            return false;
        }
        Seg g;
        g.path = f;
        g.offset = h.header_size;
        g.t0 = N_;
        g.n = n;
        g.type = h.data_type;
        g.bpe = h.bytes_per_entry;
        g.fd = ::open(f.c_str(), O_RDONLY);
        if (g.fd < 0) {
            err = "cannot open " + f;
            return false;
        }
        type_ = (M_ < 0 || type_ == h.data_type) ? h.data_type : 0;
        segs_.push_back(g);
        M_ = m;
        N_ += n;
    }
    return true;
}

bool RowReader::read(int64_t t0, int64_t nt, int32_t as_type, void* dst, std::string& err) {
    if (t0 < 0 || nt < 0 || t0 + nt > N_) {
        err = "read outside the recording";
        return false;
    }
    if (as_type != kFloat32 && !(as_type == kInt16 && type_ == kInt16)) {
        err = "unsupported conversion for " + std::to_string(as_type);
        return false;
    }
    const size_t out_bpe = as_type == kFloat32 ? 4 : 2;
    for (const Seg& g : segs_) {
        const int64_t a = std::max(t0, g.t0), b = std::min(t0 + nt, g.t0 + g.n);
        if (a >= b) continue;
        const int64_t count = (b - a) * M_;
        const int64_t off = g.offset + (a - g.t0) * M_ * g.bpe;
        char* out = static_cast<char*>(dst) + (size_t)((a - t0) * M_) * out_bpe;
        if (g.type == as_type) {
            const int fd = g.fd;
            if (!in_parts((size_t)count * out_bpe, 8,
                          [&](size_t x, size_t y) { return pread_all(fd, out + x, y - x, off + (int64_t)x); })) {
                err = "short read from " + g.path;
                return false;
            }
            continue;
        }
        // other types go through a block buffer, converted as mdaReadData does
        const int64_t block = 1 << 20;
        tmp_.resize((size_t)(block * g.bpe));
        float* of = reinterpret_cast<float*>(out);
        for (int64_t i = 0; i < count; i += block) {
            const int64_t m = std::min(block, count - i);
            if (!pread_all(g.fd, tmp_.data(), (size_t)(m * g.bpe), off + i * g.bpe)) {
                err = "short read from " + g.path;
                return false;
            }
            switch (g.type) {
                case kUint8: convert(reinterpret_cast<const uint8_t*>(tmp_.data()), of + i, m); break;
                case kFloat32: convert(reinterpret_cast<const float*>(tmp_.data()), of + i, m); break;
                case kInt16: convert(reinterpret_cast<const int16_t*>(tmp_.data()), of + i, m); break;
                case kInt32: convert(reinterpret_cast<const int32_t*>(tmp_.data()), of + i, m); break;
                case kUint16: convert(reinterpret_cast<const uint16_t*>(tmp_.data()), of + i, m); break;
                case kFloat64: convert(reinterpret_cast<const double*>(tmp_.data()), of + i, m); break;
                default: err = "unsupported data type"; return false;
            }
        }
    }
    return true;
}

RowWriter::~RowWriter() {
    if (fd_ >= 0) {
        ::close(fd_);
        std::remove(tmp_.c_str());
    }
}

bool RowWriter::open(const std::string& path, int32_t data_type, int64_t M, int64_t N, std::string& err) {
    path_ = path;
    tmp_ = path + ".tmp";
    M_ = M;
    N_ = N;
    bpe_ = bytes_per_entry(data_type);
    std::remove(path.c_str());
    fd_ = ::open(tmp_.c_str(), O_RDWR | O_CREAT | O_TRUNC, 0644);
    if (fd_ < 0) {
        err = "cannot open " + tmp_ + " for writing";
        return false;
    }
    const bool use64 = (M > 2e9) || (N > 2e9);
    unsigned char hdr[28];
    const int32_t h3[3] = {data_type, (int32_t)bpe_, use64 ? -2 : 2};
    std::memcpy(hdr, h3, 12);
    if (use64) {
        const int64_t d[2] = {M, N};
        std::memcpy(hdr + 12, d, 16);
        header_ = 28;
    } else {
        const int32_t d[2] = {(int32_t)M, (int32_t)N};
        std::memcpy(hdr + 12, d, 8);
        header_ = 20;
    }
    if (!pwrite_all(fd_, hdr, (size_t)header_, 0) || ::ftruncate(fd_, (off_t)(header_ + M * N * bpe_)) != 0) {
        err = "cannot size " + tmp_;
        return false;
    }
    return true;
}

bool RowWriter::write(int64_t t0, int64_t nt, const void* src, std::string& err) {
    if (fd_ < 0 || t0 < 0 || nt < 0 || t0 + nt > N_) {
        err = "write outside the output";
        return false;
    }
    const int64_t off = header_ + t0 * M_ * bpe_;
    const char* p = static_cast<const char*>(src);
    const int fd = fd_;
    if (!in_parts((size_t)(nt * M_ * bpe_), 4,
                  [&](size_t x, size_t y) { return pwrite_all(fd, p + x, y - x, off + (int64_t)x); })) {
        err = "write failed for " + tmp_;
        return false;
    }
    return true;
}

bool RowWriter::commit(std::string& err) {
    const int fd = fd_;
    fd_ = -1;
    if (fd < 0 || ::close(fd) != 0) {
        std::remove(tmp_.c_str());
        err = "write failed for " + tmp_;
        return false;
    }
    if (std::rename(tmp_.c_str(), path_.c_str()) != 0) {
        err = "cannot rename " + tmp_ + " to " + path_;
        return false;
    }
    return true;
}

}  // namespace ms3io
