// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// Out-of-line parts of the Qt subset in qtshim.h (file operations,
// directory listings), TextFile (declared by the reference's
// common/textfile.h), and the FFTW interface of fftw3.h over oracle/fft_ref.hpp.
#include <dirent.h>
#include <sys/stat.h>
#include <unistd.h>

#include <memory>
#include <mutex>

#include "../fft_ref.hpp"
#include "fftw3.h"
#include "qtshim.h"
#include "textfile.h"

bool QFile::exists(const QString& p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0;
}
bool QFile::remove(const QString& p) { return ::unlink(p.c_str()) == 0; }
bool QFile::rename(const QString& a, const QString& b) {
    if (exists(b)) return false;  // QFile::rename does not overwrite
    return ::rename(a.c_str(), b.c_str()) == 0;
}
bool QFile::copy(const QString& a, const QString& b) {
    if (exists(b)) return false;  // QFile::copy does not overwrite
    FILE* in = std::fopen(a.c_str(), "rb");
    if (!in) return false;
    FILE* out = std::fopen(b.c_str(), "wb");
    if (!out) {
        std::fclose(in);
        return false;
    }
    std::vector<char> buf(1 << 20);
    bool ok = true;
    for (;;) {
        const size_t n = std::fread(buf.data(), 1, buf.size(), in);
        if (n == 0) break;
        if (std::fwrite(buf.data(), 1, n, out) != n) {
            ok = false;
            break;
        }
    }
    std::fclose(in);
    ok = (std::fclose(out) == 0) && ok;
    return ok;
}
bool QFile::open(int mode) {
    close();
    f_ = std::fopen(path_.c_str(), (mode & WriteOnly) ? ((mode & ReadOnly) ? "r+b" : "wb") : "rb");
    return f_ != nullptr;
}
void QFile::close() {
    if (f_) std::fclose(f_);
    f_ = nullptr;
}
QByteArray QFile::readAll() {
    QByteArray r;
    if (!f_) return r;
    char buf[65536];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f_)) > 0) r.append(buf, n);
    return r;
}
qint64 QFile::write(const QByteArray& b) {
    if (!f_) return -1;
    return (qint64)std::fwrite(b.data(), 1, b.size(), f_);
}

bool QFileInfo::isDir() const {
    struct stat st;
    return ::stat(path_.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}
bool QFileInfo::exists() const { return QFile::exists(path_); }
QString QFileInfo::fileName() const {
    const size_t k = path_.rfind('/');
    return k == std::string::npos ? path_ : QString(path_.substr(k + 1));
}
QString QFileInfo::path() const {
    const size_t k = path_.rfind('/');
    return k == std::string::npos ? QString(".") : QString(path_.substr(0, k));
}
QString QFileInfo::suffix() const {
    const QString f = fileName();
    const size_t k = f.rfind('.');
    return k == std::string::npos ? QString() : QString(f.substr(k + 1));
}
QString QFileInfo::completeSuffix() const {
    const QString f = fileName();
    const size_t k = f.find('.');
    return k == std::string::npos ? QString() : QString(f.substr(k + 1));
}
QString QFileInfo::baseName() const {
    const QString f = fileName();
    const size_t k = f.find('.');
    return k == std::string::npos ? f : QString(f.substr(0, k));
}
qint64 QFileInfo::size() const {
    struct stat st;
    return ::stat(path_.c_str(), &st) == 0 ? (qint64)st.st_size : 0;
}

QStringList QDir::entryList(int filters, int) const {
    QStringList out;
    DIR* d = ::opendir(path_.c_str());
    if (!d) return out;
    while (struct dirent* e = ::readdir(d)) {
        const std::string name = e->d_name;
        if (name == "." || name == "..") continue;
        const bool dir = QFileInfo(path_ + "/" + name).isDir();
        if ((dir && (filters & Dirs)) || (!dir && (filters & Files))) out.push_back(QString(name));
    }
    ::closedir(d);
    std::sort(out.begin(), out.end());
    return out;
}
QStringList QDir::entryList(const QStringList&, int filters, int sort) const { return entryList(filters, sort); }

QString TextFile::read(const QString& fname, QTextCodec*) {
    QFile f(fname);
    if (!f.open(QFile::ReadOnly)) return QString();
    return QString(f.readAll());
}
bool TextFile::write(const QString& fname, const QString& txt, QTextCodec*) {
    QFile f(fname);
    if (!f.open(QFile::WriteOnly)) return false;
    return f.write(QByteArray(txt)) == (qint64)txt.size();
}
bool TextFile::write_single_try(const QString& fname, const QString& txt, QTextCodec* c) { return write(fname, txt, c); }

// ------------------------------------------------------------ FFTW interface

struct ms3ref_fftwf_plan {
    std::unique_ptr<ms3ref::BatchedFft> fft;
    int64_t n = 0;
    int howmany = 0;
    float* in = nullptr;
    float* out = nullptr;
    int istride = 1, idist = 1, ostride = 1, odist = 1;
};

void* fftwf_malloc(size_t n) { return std::malloc(n ? n : 1); }
void fftwf_free(void* p) { std::free(p); }
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int) {}
void fftwf_cleanup_threads(void) {}

fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany, fftwf_complex* in, const int*, int istride,
                               int idist, fftwf_complex* out, const int*, int ostride, int odist, int sign,
                               unsigned) {
    if (rank != 1 || howmany < 1) return nullptr;
    auto* p = new ms3ref_fftwf_plan;
    p->fft.reset(new ms3ref::BatchedFft(n[0], sign));
    p->n = n[0];
    p->howmany = howmany;
    p->in = reinterpret_cast<float*>(in);
    p->out = reinterpret_cast<float*>(out);
    p->istride = istride;
    p->idist = idist;
    p->ostride = ostride;
    p->odist = odist;
    return p;
}

// Gathers the transforms into the interleaved layout of BatchedFft (element
// j of transform b at j * howmany + b), transforms, scatters to `out`.
void fftwf_execute(const fftwf_plan p) {
    const int64_t L = p->n, H = p->howmany;
    const bool direct = p->istride == H && p->idist == 1 && p->ostride == H && p->odist == 1;
    std::vector<float> buf(direct ? 0 : (size_t)(2 * L * H)), work((size_t)(2 * L * H));
    float* data = direct ? p->out : buf.data();
    if (direct) {
        if (p->out != p->in) std::memcpy(p->out, p->in, sizeof(float) * 2 * L * H);
    } else {
        for (int64_t b = 0; b < H; b++)
            for (int64_t j = 0; j < L; j++) {
                const float* s = p->in + 2 * (j * p->istride + b * p->idist);
                data[2 * (j * H + b)] = s[0];
                data[2 * (j * H + b) + 1] = s[1];
            }
    }
    p->fft->execute(data, work.data(), H);
    if (!direct) {
        for (int64_t b = 0; b < H; b++)
            for (int64_t j = 0; j < L; j++) {
                float* d = p->out + 2 * (j * p->ostride + b * p->odist);
                d[0] = data[2 * (j * H + b)];
                d[1] = data[2 * (j * H + b) + 1];
            }
    }
}

void fftwf_destroy_plan(fftwf_plan p) { delete p; }
