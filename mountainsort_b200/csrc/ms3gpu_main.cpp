// ms3gpu.mp -- MountainLab processor executable for ms3.bandpass_filter,
// ms3.whiten, ms3.compute_whitening_matrix, ms3.apply_whitening_matrix,
// ms3.whiten_clips and ms3.mask_out_artifacts, backed by libms3gpu (CUDA,
// sm_100a).
//
// Same command-line protocol as the reference's ms3.mp
// (packages/ms3/mountainsort3_main.cpp:379-821):
//   ms3gpu.mp spec [name]
//   ms3gpu.mp requirements <name> --key=value ...
//   ms3gpu.mp ms3.bandpass_filter --timeseries=in.mda --timeseries_out=out.mda
//       --samplerate=.. --freq_min=.. --freq_max=.. [--freq_wid=1000]
//       [--quantization_unit=0] [--subsample_factor=1] [--_request_num_threads=T]
//   ms3gpu.mp ms3.whiten --timeseries=in.mda --timeseries_out=out.mda [--quantization_unit=0]
// Exit status 0 on success, -1 (255) on failure or for an unknown processor.
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "mdaio.h"
#include "ms3gpu.h"

namespace {

// CLParams (packages/ms3/common/clparams.cpp:20-77): "--name=value" or
// "--name value"; everything else is an unnamed parameter.  A name given
// more than once becomes a list (:55-68): `lists` keeps every value in
// order, `named` the last one.
struct CLParams {
    std::map<std::string, std::string> named;
    std::map<std::string, std::vector<std::string>> lists;
    std::vector<std::string> unnamed;
    bool success = true;
    std::string error;
    CLParams(int argc, char** argv) {
        for (int i = 1; i < argc; i++) {
            std::string s = argv[i];
            if (s.rfind("--", 0) == 0) {
                std::string name, val;
                const size_t eq = s.find('=');
                if (eq != std::string::npos) {
                    name = s.substr(2, eq - 2);
                    val = s.substr(eq + 1);
                } else {
                    name = s.substr(2);
                    if (i + 1 < argc && std::string(argv[i + 1]).rfind("--", 0) != 0) val = argv[++i];
                }
                if (name.empty()) {
                    success = false;
                    error = "Problem with parameter: " + s;
                    return;
                }
                named[name] = val;
                lists[name].push_back(val);
            } else {
                unnamed.push_back(s);
            }
        }
    }
    bool has(const std::string& k) const { return named.count(k) > 0; }
    std::string str(const std::string& k) const {
        auto it = named.find(k);
        return it == named.end() ? std::string() : it->second;
    }
    // QVariant::toDouble(): 0 for a missing or non-numeric value
    double num(const std::string& k, double dflt) const {
        auto it = named.find(k);
        if (it == named.end()) return dflt;
        char* end = nullptr;
        const double v = std::strtod(it->second.c_str(), &end);
        return (end && end != it->second.c_str()) ? v : 0.0;
    }
};

std::string exe_path() {
    char buf[4096];
    const ssize_t n = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
    if (n <= 0) return "ms3gpu.mp";
    buf[n] = 0;
    return buf;
}

std::string json_escape(const std::string& s) {
    std::string o;
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o;
}

struct Param {
    std::string name;
    bool optional;
    std::string default_json;  // empty: no default
};

// ProcessorSpec::get_spec (mountainsort3_main.cpp:965-983); keys sorted as
// QJsonObject serialises them.
std::string processor_spec(const std::string& name, const std::string& version,
                           const std::vector<std::string>& inputs, const std::vector<std::string>& outputs,
                           const std::vector<Param>& params, const std::string& ind,
                           bool can_return_requirements = true) {
    const std::string exe = exe_path();
    auto files = [&](const std::vector<std::string>& v) {
        std::string o = "[\n";
        for (size_t i = 0; i < v.size(); i++) {
            o += ind + "        {\n" + ind + "            \"description\": \"\",\n" + ind + "            \"name\": \"" +
                 v[i] + "\",\n" + ind + "            \"optional\": false\n" + ind + "        }";
            o += (i + 1 < v.size()) ? ",\n" : "\n";
        }
        return o + ind + "    ]";
    };
    std::string ps = "[\n";
    for (size_t i = 0; i < params.size(); i++) {
        const Param& p = params[i];
        ps += ind + "        {\n";
        if (!p.default_json.empty()) ps += ind + "            \"default_value\": " + p.default_json + ",\n";
        ps += ind + "            \"description\": \"\",\n" + ind + "            \"name\": \"" + p.name + "\",\n" + ind +
              "            \"optional\": " + (p.optional ? "true" : "false") + "\n" + ind + "        }";
        ps += (i + 1 < params.size()) ? ",\n" : "\n";
    }
    ps += ind + "    ]";
    std::string o = ind + "{\n";
    o += ind + "    \"description\": \"\",\n";
    o += ind + "    \"exe_command\": \"" + json_escape(exe) + " " + name + " $(arguments)\",\n";
    o += ind + "    \"inputs\": " + files(inputs) + ",\n";
    o += ind + "    \"name\": \"" + name + "\",\n";
    o += ind + "    \"outputs\": " + files(outputs) + ",\n";
    o += ind + "    \"parameters\": " + ps + ",\n";
    if (can_return_requirements)
        o += ind + "    \"requirements_command\": \"" + json_escape(exe) + " requirements " + name + " $(arguments)\",\n";
    o += ind + "    \"version\": \"" + version + "\"\n";
    o += ind + "}";
    return o;
}

// Registered at mountainsort3_main.cpp:146-165 (same names, versions,
// parameters and defaults).
std::string spec_bandpass(const std::string& ind) {
    return processor_spec("ms3.bandpass_filter", "0.20", {"timeseries"}, {"timeseries_out"},
                          {{"samplerate", false, ""},
                           {"freq_min", false, ""},
                           {"freq_max", false, ""},
                           {"freq_wid", true, "1000"},
                           {"quantization_unit", true, "0"},
                           {"subsample_factor", true, "1"}},
                          ind);
}
std::string spec_whiten(const std::string& ind) {
    return processor_spec("ms3.whiten", "0.1", {"timeseries"}, {"timeseries_out"},
                          {{"quantization_unit", true, "0"}}, ind);
}
// mountainsort3_main.cpp:166-189 (no requirements command for these)
std::string spec_compute_whitening_matrix(const std::string& ind) {
    return processor_spec("ms3.compute_whitening_matrix", "0.11", {"timeseries_list"}, {"whitening_matrix_out"},
                          {{"channels", true, ""}}, ind, false);
}
std::string spec_whiten_clips(const std::string& ind) {
    return processor_spec("ms3.whiten_clips", "0.1", {"clips", "whitening_matrix"}, {"clips_out"},
                          {{"quantization_unit", true, "0"}}, ind, false);
}
// mountainsort3_main.cpp:343-350
std::string spec_mask_out_artifacts(const std::string& ind) {
    return processor_spec("ms3.mask_out_artifacts", "0.1", {"timeseries"}, {"timeseries_out"},
                          {{"threshold", true, "6"}, {"interval_size", true, "2000"}}, ind, false);
}
std::string spec_apply_whitening_matrix(const std::string& ind) {
    return processor_spec("ms3.apply_whitening_matrix", "0.1", {"timeseries", "whitening_matrix"},
                          {"timeseries_out"}, {{"quantization_unit", true, "0"}}, ind, false);
}

// T of the chunk-size formula: omp_get_max_threads() in the reference, set
// by --_request_num_threads (mountainsort3_main.cpp:428-434); without it,
// OpenMP's default (OMP_NUM_THREADS, else the number of hardware threads).
int geometry_threads(const CLParams& clp) {
    const int req = (int)clp.num("_request_num_threads", 0);
    if (req > 0) return req;
    const char* e = std::getenv("OMP_NUM_THREADS");
    if (e && *e) {
        const int v = std::atoi(e);
        if (v > 0) return v;
    }
    const unsigned hc = std::thread::hardware_concurrency();
    return hc ? (int)hc : 1;
}

ms3gpu_bandpass_opts bandpass_opts(const CLParams& clp) {
    // mountainsort3_main.cpp:547-557
    ms3gpu_bandpass_opts o;
    o.samplerate = clp.num("samplerate", 0);
    o.freq_min = clp.num("freq_min", 0);
    o.freq_max = clp.num("freq_max", 0);
    o.freq_wid = clp.num("freq_wid", 1000);
    o.quantization_unit = clp.num("quantization_unit", 0);
    o.subsample_factor = (int32_t)clp.num("subsample_factor", 1);
    if (!o.subsample_factor) o.subsample_factor = 1;
    o.num_threads = geometry_threads(clp);
    return o;
}

void print_requirements(double mb) { std::printf("{\n    \"peak_ram_mb\": %.17g\n}\n", mb); }

int fail(const std::string& msg) {
    std::fprintf(stderr, "ms3gpu: %s\n", msg.c_str());
    return -1;
}

int32_t precision_of(const CLParams& clp) {
    // --_precision=mixed selects the mixed form (not a reference parameter)
    return clp.str("_precision") == "mixed" ? MS3GPU_PRECISION_MIXED : MS3GPU_PRECISION_PLAIN;
}

// The processors' files as the streaming entry points read and write them:
// rows of the input (converted to float32 unless kept as int16) and rows of
// the output's .tmp file.
struct StreamFiles {
    ms3io::RowReader in;
    ms3io::RowWriter out;
    int32_t in_type = ms3io::kFloat32;
    std::string err;
};

int read_rows_cb(void* ctx, int64_t t0, int64_t nt, void* dst) {
    auto* f = static_cast<StreamFiles*>(ctx);
    return f->in.read(t0, nt, f->in_type, dst, f->err) ? 0 : 1;
}

int write_rows_cb(void* ctx, int64_t t0, int64_t nt, const void* src) {
    auto* f = static_cast<StreamFiles*>(ctx);
    return f->out.write(t0, nt, src, f->err) ? 0 : 1;
}

// --_slab_mb=<MB> sets the rows read per block (not a reference parameter;
// default 1024)
int64_t slab_bytes(const CLParams& clp) {
    const double mb = clp.num("_slab_mb", 0);
    return mb > 0 ? (int64_t)(mb * 1048576.0) : (int64_t(1) << 30);
}

ms3gpu_stream_io stream_io(StreamFiles& f, const CLParams& clp) {
    ms3gpu_stream_io io{};
    io.read = read_rows_cb;
    io.read_ctx = &f;
    io.write = write_rows_cb;
    io.write_ctx = &f;
    io.slab_bytes = (int64_t)(clp.num("_slab_mb", 0) * 1048576.0);
    return io;
}

int stream_fail(const StreamFiles& f) {
    std::string msg = ms3gpu_last_error();
    if (!f.err.empty()) msg += ": " + f.err;
    return fail(msg);
}

int run_bandpass(const CLParams& clp, bool requirements_only) {
    const std::string in = clp.str("timeseries"), out = clp.str("timeseries_out");
    ms3gpu_bandpass_opts o = bandpass_opts(clp);
    std::string err;
    if (o.freq_max == 0 && !requirements_only) {
        // p_bandpass_filter.cpp:117-119 (QFile::copy, which cannot copy a directory)
        if (ms3io::is_directory(in)) return fail("cannot copy a directory: " + in);
        if (!ms3io::copy_file(in, out, err)) return fail(err);
        return 0;
    }
    // a file, or a directory of .mda files concatenated in time (:128-131)
    int64_t M = 0, N = 0;
    int32_t dtype = 0;
    if (!ms3io::read_dims_any(in, M, N, dtype, err)) return fail(err);
    if (requirements_only) {
        double mb = 0;
        if (ms3gpu_bandpass_requirements(M, N, &o, &mb) != MS3GPU_OK) {
            std::printf("Error in processor while trying to retrieve requirements.\n");
            return -1;
        }
        print_requirements(mb);
        return 0;
    }
    int64_t Mo = 0, No = 0;
    int32_t dt = 0;
    if (ms3gpu_bandpass_output_dims(M, N, &o, &Mo, &No, &dt) != MS3GPU_OK) return fail(ms3gpu_last_error());
    std::fprintf(stderr, "ms3gpu: bandpass %lld x %lld, chunk %lld (T=%d)\n", (long long)M, (long long)N,
                 (long long)ms3gpu_bandpass_chunk_size(M, o.num_threads), o.num_threads);
    // the recording streams through the GPU in slabs of whole chunks; int16
    // recordings go to the GPU as int16 and are converted in the filter's loads
    StreamFiles f;
    if (!f.in.open(in, err)) return fail(err);
    f.in_type = f.in.data_type() == ms3io::kInt16 ? ms3io::kInt16 : ms3io::kFloat32;
    if (!f.out.open(out, dt, Mo, No, err)) return fail(err);
    const ms3gpu_stream_io io = stream_io(f, clp);
    const int32_t in_dtype = f.in_type == ms3io::kInt16 ? MS3GPU_DTYPE_INT16 : MS3GPU_DTYPE_FLOAT32;
    if (ms3gpu_bandpass_filter_stream(M, N, in_dtype, &io, &o, nullptr) != MS3GPU_OK) return stream_fail(f);
    if (!f.out.commit(err)) return fail(err);
    return 0;
}

int run_whiten(const CLParams& clp, bool requirements_only) {
    const std::string in = clp.str("timeseries"), out = clp.str("timeseries_out");
    ms3gpu_whiten_opts o;
    o.quantization_unit = clp.num("quantization_unit", 0);  // mountainsort3_main.cpp:576
    o.precision = precision_of(clp);
    std::string err;
    int64_t M = 0, N = 0;
    int32_t dtype = 0;
    if (!ms3io::read_dims_any(in, M, N, dtype, err)) return fail(err);
    if (requirements_only) {
        double mb = 0;
        if (ms3gpu_whiten_requirements(M, N, &mb) != MS3GPU_OK) {
            std::printf("Error in processor while trying to retrieve requirements.\n");
            return -1;
        }
        print_requirements(mb);
        return 0;
    }
    // two passes over the input, as the reference reads it (p_whiten.cpp:64-206)
    StreamFiles f;
    if (!f.in.open(in, err)) return fail(err);
    const bool i16 = o.quantization_unit > 0;
    if (!f.out.open(out, i16 ? ms3io::kInt16 : ms3io::kFloat32, M, N, err)) return fail(err);
    const ms3gpu_stream_io io = stream_io(f, clp);
    if (ms3gpu_whiten_stream(M, N, &io, &o, nullptr) != MS3GPU_OK) return stream_fail(f);
    if (!f.out.commit(err)) return fail(err);
    return 0;
}

// A whitening matrix file (Mda WW(path): any dtype, read as double), M x M.
bool read_whitening_matrix(const std::string& path, int64_t M, std::vector<double>& W, std::string& err) {
    std::vector<int64_t> dims;
    if (!ms3io::read_array_f64(path, dims, W, err)) return false;
    const int64_t n1 = dims.size() > 0 ? dims[0] : 1, n2 = dims.size() > 1 ? dims[1] : 1;
    if (n1 != M || n2 != M || (int64_t)W.size() != M * M) {
        err = "whitening matrix " + path + " is not " + std::to_string(M) + " x " + std::to_string(M);
        return false;
    }
    return true;
}

// p_compute_whitening_matrix (p_whiten.cpp:208-298) with the arguments of
// mountainsort3_main.cpp:594-600.
int run_compute_whitening_matrix(const CLParams& clp) {
    auto it = clp.lists.find("timeseries_list");
    if (it == clp.lists.end() || it->second.empty()) return fail("timeseries_list is empty");
    const std::string out = clp.str("whitening_matrix_out");
    std::vector<int32_t> channels;
    {
        // split(",", SkipEmptyParts) then toInt (0 for a non-number)
        const std::string cs = clp.str("channels");
        size_t a = 0;
        while (a <= cs.size()) {
            size_t b = cs.find(',', a);
            if (b == std::string::npos) b = cs.size();
            if (b > a) channels.push_back((int32_t)std::atoi(cs.substr(a, b - a).c_str()));
            a = b + 1;
        }
    }
    // The recordings are read block by block: each block's x x^T sum over the
    // selected channels (ms3gpu_whiten_covariance_sum) is added into an FP64
    // total, divided by (total timepoints - 1) as the reference divides
    // (p_whiten.cpp:270-280), then the whitening matrix of that XXt.
    std::string err;
    int64_t M = -1;
    std::vector<ms3io::RowReader> readers(it->second.size());
    for (size_t i = 0; i < it->second.size(); i++) {
        if (!readers[i].open(it->second[i], err)) return fail(err);
        if (M >= 0 && readers[i].M() != M) return fail("the recordings of timeseries_list differ in channel count");
        M = readers[i].M();
    }
    for (int32_t c : channels)
        if (c < 1 || c > M)
            return fail("channel " + std::to_string(c) + " outside 1.." + std::to_string(M) + " in channels");
    const int64_t M2 = channels.empty() ? M : (int64_t)channels.size();
    std::vector<double> total((size_t)(M2 * M2), 0.0), part((size_t)(M2 * M2));
    int64_t Ntot = 0;
    const int64_t rows = std::max<int64_t>(1, slab_bytes(clp) / std::max<int64_t>(1, 4 * M));
    std::vector<float> xb, sb;
    for (ms3io::RowReader& r : readers) {
        const int64_t Ni = r.N();
        for (int64_t t = 0; t < Ni && M2 > 0; t += rows) {
            const int64_t nt = std::min(rows, Ni - t);
            xb.resize((size_t)(nt * M));
            if (!r.read(t, nt, ms3io::kFloat32, xb.data(), err)) return fail(err);
            const float* blk = xb.data();
            if (!channels.empty()) {
                sb.resize((size_t)(nt * M2));
                for (int64_t k = 0; k < nt; k++)
                    for (int64_t j = 0; j < M2; j++) sb[(size_t)(k * M2 + j)] = xb[(size_t)(k * M + channels[(size_t)j] - 1)];
                blk = sb.data();
            }
            if (ms3gpu_whiten_covariance_sum(blk, M2, nt, part.data(), nullptr) != MS3GPU_OK)
                return fail(ms3gpu_last_error());
            for (size_t e = 0; e < total.size(); e++) total[e] += part[e];
        }
        Ntot += Ni;
    }
    if (Ntot > 1)
        for (double& v : total) v /= (double)(Ntot - 1);
    std::vector<double> W((size_t)(M2 * M2));
    if (M2 > 0 && ms3gpu_whitening_matrix(total.data(), M2, W.data(), nullptr, nullptr, nullptr) != MS3GPU_OK)
        return fail(ms3gpu_last_error());
    // Mda::write64 (float64)
    if (!ms3io::write_array(out, ms3io::kFloat64, {M2, M2}, W.data(), err)) return fail(err);
    return 0;
}

// p_apply_whitening_matrix (p_whiten.cpp:347-417)
int run_apply_whitening_matrix(const CLParams& clp) {
    const std::string in = clp.str("timeseries"), wpath = clp.str("whitening_matrix"), out = clp.str("timeseries_out");
    const double q = clp.num("quantization_unit", 0);
    std::string err;
    ms3io::RowReader rd;
    if (!rd.open(in, err)) return fail(err);
    const int64_t M = rd.M(), N = rd.N();
    std::vector<double> W;
    if (!read_whitening_matrix(wpath, M, W, err)) return fail(err);
    const bool i16 = q > 0;
    ms3io::RowWriter wr;
    if (!wr.open(out, i16 ? ms3io::kInt16 : ms3io::kFloat32, M, N, err)) return fail(err);
    // block by block: the apply is per timepoint, so the values are those of one call
    const int64_t rows = std::max<int64_t>(1, slab_bytes(clp) / std::max<int64_t>(1, 4 * M));
    std::vector<float> xb;
    std::vector<unsigned char> yb;
    for (int64_t t = 0; t < N && M > 0; t += rows) {
        const int64_t nt = std::min(rows, N - t);
        xb.resize((size_t)(nt * M));
        yb.resize((size_t)(nt * M) * (i16 ? 2 : 4));
        if (!rd.read(t, nt, ms3io::kFloat32, xb.data(), err)) return fail(err);
        if (ms3gpu_apply_whitening_matrix(xb.data(), M, nt, W.data(), q, precision_of(clp), yb.data(), nullptr) !=
            MS3GPU_OK)
            return fail(ms3gpu_last_error());
        if (!wr.write(t, nt, yb.data(), err)) return fail(err);
    }
    if (!wr.commit(err)) return fail(err);
    return 0;
}

// p_whiten_clips (p_whiten.cpp:300-345): clips M x T x L
int run_whiten_clips(const CLParams& clp) {
    const std::string in = clp.str("clips"), wpath = clp.str("whitening_matrix"), out = clp.str("clips_out");
    const double q = clp.num("quantization_unit", 0);
    std::string err;
    std::vector<int64_t> dims;
    std::vector<float> C;
    if (!ms3io::read_array_f32(in, dims, C, err)) return fail(err);
    const int64_t M = dims.size() > 0 ? dims[0] : 1, T = dims.size() > 1 ? dims[1] : 1;
    const int64_t L = (M * T) ? (int64_t)C.size() / (M * T) : 0;
    std::vector<double> W;
    if (!read_whitening_matrix(wpath, M, W, err)) return fail(err);
    const bool i16 = q > 0;
    std::vector<unsigned char> Y((size_t)(M * T * L) * (i16 ? 2 : 4));
    if (ms3gpu_whiten_clips(C.data(), M, T, L, W.data(), q, precision_of(clp), Y.data(), nullptr) != MS3GPU_OK)
        return fail(ms3gpu_last_error());
    if (!ms3io::write_array(out, i16 ? ms3io::kInt16 : ms3io::kFloat32, {M, T, L}, Y.data(), err)) return fail(err);
    return 0;
}

// p_mask_out_artifacts (p_mask_out_artifacts.cpp:24-104) with the arguments
// of mountainsort3_main.cpp:782-787 (interval_size read as a double, then
// truncated to an integer)
int run_mask_out_artifacts(const CLParams& clp) {
    const std::string in = clp.str("timeseries"), out = clp.str("timeseries_out");
    const double threshold = clp.num("threshold", 0);
    const int64_t interval_size = (int64_t)clp.num("interval_size", 0);
    if (!threshold || !interval_size) {
        std::printf("Problem with input parameters. Either threshold or interval_size is zero.\n");
        return -1;
    }
    std::string err;
    // two passes over the input in blocks of whole intervals (the norms,
    // then the masked copy), as the reference reads it twice
    StreamFiles f;
    if (!f.in.open(in, err)) return fail(err);
    const int64_t M = f.in.M(), N = f.in.N();
    if (!f.out.open(out, ms3io::kFloat32, M, N, err)) return fail(err);
    const ms3gpu_stream_io io = stream_io(f, clp);
    int64_t kept = 0;
    if (ms3gpu_mask_out_artifacts_stream(M, N, threshold, interval_size, &io, &kept, nullptr) != MS3GPU_OK)
        return stream_fail(f);
    if (!f.out.commit(err)) return fail(err);
    const int64_t nint = N / interval_size;
    if (nint > 0) std::printf("Using %.2f%% of all timepoints\n", kept * 100.0 / (double)(nint * interval_size));
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    CLParams clp(argc, argv);
    if (!clp.success) return fail(clp.error);
    const std::string arg1 = clp.unnamed.size() > 0 ? clp.unnamed[0] : "";
    const std::string arg2 = clp.unnamed.size() > 1 ? clp.unnamed[1] : "";
    if (arg1 == "spec") {
        std::string (*const specs[])(const std::string&) = {spec_bandpass, spec_whiten,
                                                             spec_compute_whitening_matrix, spec_whiten_clips,
                                                             spec_apply_whitening_matrix, spec_mask_out_artifacts};
        const char* const names[] = {"ms3.bandpass_filter", "ms3.whiten", "ms3.compute_whitening_matrix",
                                     "ms3.whiten_clips", "ms3.apply_whitening_matrix", "ms3.mask_out_artifacts"};
        const size_t nspec = sizeof(names) / sizeof(names[0]);
        if (arg2.empty()) {
            std::string all;
            for (size_t i = 0; i < nspec; i++) all += (i ? ",\n" : "") + specs[i]("        ");
            std::printf("{\n    \"processors\": [\n%s\n    ]\n}\n\n", all.c_str());
            return 0;
        }
        for (size_t i = 0; i < nspec; i++) {
            if (arg2 == names[i]) {
                std::printf("%s\n\n", specs[i]("").c_str());
                return 0;
            }
        }
        std::printf("{}\n");
        return -1;
    }
    bool requirements_only = false;
    std::string pname = arg1;
    if (arg1 == "requirements") {
        pname = arg2;
        requirements_only = true;
    }
    if (pname == "ms3.bandpass_filter") return run_bandpass(clp, requirements_only);
    if (pname == "ms3.whiten") return run_whiten(clp, requirements_only);
    if (!requirements_only) {
        if (pname == "ms3.compute_whitening_matrix") return run_compute_whitening_matrix(clp);
        if (pname == "ms3.apply_whitening_matrix") return run_apply_whitening_matrix(clp);
        if (pname == "ms3.whiten_clips") return run_whiten_clips(clp);
        if (pname == "ms3.mask_out_artifacts") return run_mask_out_artifacts(clp);
    }
    std::fprintf(stderr, "Unexpected processor name: %s\n", pname.c_str());
    return -1;
}
