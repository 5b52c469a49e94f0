// .mda file I/O for the ms3gpu.mp processor executable.
//
// Format (packages/ms3/mda/mdaio.cpp:60-203): int32 data type code, int32
// bytes per entry, int32 number of dims (negative: the dims are int64), the
// dims, then the data column-major.  Timeseries are read as float32 with the
// reference's conversions (mdaReadData, mdaio.cpp:205-230); outputs are
// written to `path.tmp` and renamed when complete (mda/diskwritemda.cpp:57-149).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ms3io {

constexpr int32_t kUint8 = -2, kFloat32 = -3, kInt16 = -4, kInt32 = -5, kUint16 = -6, kFloat64 = -7,
                  kUint32 = -8;

struct MdaHeader {
    int32_t data_type = 0;
    int32_t bytes_per_entry = 0;
    std::vector<int64_t> dims;
    int64_t header_size = 0;
    bool uses64bitdims = false;
};

int bytes_per_entry(int32_t data_type);

// Parses the header of `path`; false with a message on error.
bool read_header(const std::string& path, MdaHeader& h, std::string& err);

// Reads an M x N (first two dims) timeseries converted to float32.
bool read_timeseries_f32(const std::string& path, int64_t& M, int64_t& N, std::vector<float>& data,
                         std::string& err);

// Writes an M x N array of `data_type` (kFloat32 or kInt16) from `data`.
bool write_timeseries(const std::string& path, int32_t data_type, int64_t M, int64_t N, const void* data,
                      std::string& err);

// Every entry of an N-dimensional array, converted to float32 / float64.
bool read_array_f32(const std::string& path, std::vector<int64_t>& dims, std::vector<float>& data,
                    std::string& err);
bool read_array_f64(const std::string& path, std::vector<int64_t>& dims, std::vector<double>& data,
                    std::string& err);

// Writes an N-dimensional array of `data_type` (via path.tmp + rename).
bool write_array(const std::string& path, int32_t data_type, const std::vector<int64_t>& dims, const void* data,
                 std::string& err);

bool is_directory(const std::string& path);

// A timeseries input as the reference's DiskReadMda32 opens it
// (mda/diskreadmda32.cpp:234-237, 283-288): a file, or a directory whose
// .mda files are concatenated along time.
bool input_files(const std::string& path, std::vector<std::string>& files, std::string& err);
// M, total N and the common data type (0 when the files' types differ).
bool read_dims_any(const std::string& path, int64_t& M, int64_t& N, int32_t& data_type, std::string& err);
bool read_timeseries_any_f32(const std::string& path, int64_t& M, int64_t& N, std::vector<float>& data,
                             std::string& err);
// An int16 file's entries as they are (no conversion).
bool read_timeseries_i16(const std::string& path, int64_t& M, int64_t& N, std::vector<int16_t>& data,
                         std::string& err);

// Timepoint rows of a timeseries input (a file, or a directory's .mda files
// concatenated in time) read block by block, as DiskReadMda32::readChunk
// reads them (mda/diskreadmda32.cpp:615-661).  Entries are converted to
// float32 as mdaReadData converts them (mdaio.cpp:205-230), or kept as int16
// when every file is int16.
class RowReader {
public:
    RowReader() = default;
    ~RowReader();
    RowReader(const RowReader&) = delete;
    RowReader& operator=(const RowReader&) = delete;
    bool open(const std::string& path, std::string& err);
    int64_t M() const { return M_; }
    int64_t N() const { return N_; }
    // the files' common data type, 0 when they differ
    int32_t data_type() const { return type_; }
    // timepoints [t0, t0 + nt) (M entries each) into dst as `as_type`:
    // kFloat32, or kInt16 when data_type() is kInt16
    bool read(int64_t t0, int64_t nt, int32_t as_type, void* dst, std::string& err);

private:
    struct Seg {
        std::string path;
        int fd = -1;
        int64_t offset = 0, t0 = 0, n = 0;
        int32_t type = 0;
        int bpe = 0;
    };
    std::vector<Seg> segs_;
    int64_t M_ = 0, N_ = 0;
    int32_t type_ = 0;
    std::vector<unsigned char> tmp_;
};

// An M x N timeseries written block by block into `path.tmp`, which is sized
// in full when opened (rows never written read as zero, like the reference's
// preallocated file) and renamed to `path` by commit()
// (mda/diskwritemda.cpp:57-149, 255-265).  Without commit() the .tmp file is
// removed.
class RowWriter {
public:
    RowWriter() = default;
    ~RowWriter();
    RowWriter(const RowWriter&) = delete;
    RowWriter& operator=(const RowWriter&) = delete;
    bool open(const std::string& path, int32_t data_type, int64_t M, int64_t N, std::string& err);
    // timepoints [t0, t0 + nt), M entries each, of the output's data type
    bool write(int64_t t0, int64_t nt, const void* src, std::string& err);
    bool commit(std::string& err);

private:
    int fd_ = -1;
    std::string path_, tmp_;
    int64_t M_ = 0, N_ = 0, header_ = 0;
    int bpe_ = 0;
};

// Byte copy that, like QFile::copy, refuses to overwrite an existing file.
bool copy_file(const std::string& src, const std::string& dst, std::string& err);

}  // namespace ms3io
