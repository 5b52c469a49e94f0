// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// The smallest part of the Qt 5 Core API that the reference's ms3
// preprocessing sources use (packages/ms3/p_bandpass_filter.cpp,
// p_whiten.cpp, pca.cpp, common/mlcompute.cpp and the mda/ I/O classes), so
// that those files compile here unchanged without Qt.  Only what those files
// call is provided; the semantics follow Qt's documentation for the calls
// they make (implicit sharing of QSharedDataPointer with detach on non-const
// access, QString::arg place markers, split with SkipEmptyParts, QFile's
// static file operations).  Written for this purpose; no Qt code is used.
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <numeric>
#include <type_traits>
#include <sstream>
#include <string>
#include <vector>

typedef std::intptr_t qintptr;
typedef long long qint64;
typedef unsigned long long quint64;
#define Q_UNUSED(x) (void)(x);
#define foreach(decl, container) for (decl : container)

template <class T>
inline const T& qMin(const T& a, const T& b) { return (b < a) ? b : a; }
template <class T>
inline const T& qMax(const T& a, const T& b) { return (a < b) ? b : a; }

class QTextCodec;
class QVariant;
class QJsonValue;

// ------------------------------------------------------------ containers

inline int qrand() { return std::rand(); }
inline void qsrand(unsigned s) { std::srand(s); }

template <class T>
class QList : public std::vector<T> {
public:
    QList() {}
    QList(std::initializer_list<T> l) : std::vector<T>(l) {}
    template <class I, class = typename std::enable_if<std::is_integral<I>::value>::type>
    explicit QList(I n) : std::vector<T>((size_t)n) {}
    template <class I, class = typename std::enable_if<std::is_integral<I>::value>::type>
    QList(I n, const T& v) : std::vector<T>((size_t)n, v) {}
    template <class S>
    S join(const S& sep) const {  // QList<QString>::join
        S r;
        for (size_t i = 0; i < this->size(); i++) {
            if (i) r += sep;
            r += (*this)[i];
        }
        return r;
    }
    template <class S = T>
    S join(const char* sep) const { return join(S(sep)); }
    int count() const { return (int)this->size(); }
    int length() const { return (int)this->size(); }
    bool isEmpty() const { return this->empty(); }
    void append(const T& v) { this->push_back(v); }
    void append(const QList<T>& o) { this->insert(this->end(), o.begin(), o.end()); }
    QList& operator<<(const T& v) { this->push_back(v); return *this; }
    QList& operator<<(const QList<T>& o) { append(o); return *this; }
    const T& at(qintptr i) const { return (*this)[(size_t)i]; }
    T value(qintptr i) const { return (i < 0 || i >= (qintptr)this->size()) ? T() : (*this)[(size_t)i]; }
    T value(qintptr i, const T& d) const { return (i < 0 || i >= (qintptr)this->size()) ? d : (*this)[(size_t)i]; }
    // An index outside the list lands in a scratch slot instead of memory
    // next to the list: p_mask_out_artifacts.cpp writes use_it[i - 1] for
    // i == 0, which is undefined behaviour in the reference; here the write
    // is dropped, as the oracle's restatement drops it.
    T& operator[](qintptr i) {
        if (i < 0 || i >= (qintptr)this->size()) {
            static thread_local T scratch;
            scratch = T();
            return scratch;
        }
        return std::vector<T>::operator[]((size_t)i);
    }
    const T& operator[](qintptr i) const { return std::vector<T>::operator[]((size_t)i); }
    typename std::vector<T>::const_iterator constBegin() const { return this->begin(); }
    typename std::vector<T>::const_iterator constEnd() const { return this->end(); }
    bool contains(const T& v) const { return std::find(this->begin(), this->end(), v) != this->end(); }
    int indexOf(const T& v) const {
        auto it = std::find(this->begin(), this->end(), v);
        return it == this->end() ? -1 : (int)(it - this->begin());
    }
    const T& first() const { return this->front(); }
    const T& last() const { return this->back(); }
};

template <class T>
class QVector : public QList<T> {
public:
    QVector() {}
    QVector(std::initializer_list<T> l) : QList<T>(l) {}
    template <class I, class = typename std::enable_if<std::is_integral<I>::value>::type>
    explicit QVector(I n) : QList<T>((size_t)n) {}
    template <class I, class = typename std::enable_if<std::is_integral<I>::value>::type>
    QVector(I n, const T& v) : QList<T>((size_t)n, v) {}
    void fill(const T& v) { std::fill(this->begin(), this->end(), v); }
};

template <class T>
inline void qSort(QVector<T>& v) { std::sort(v.begin(), v.end()); }
template <class T>
inline void qSort(QList<T>& v) { std::sort(v.begin(), v.end()); }

// ------------------------------------------------------------ strings

class QByteArray : public std::string {
public:
    using std::string::string;
    QByteArray() {}
    QByteArray(const std::string& s) : std::string(s) {}
    QByteArray(const char* p, qintptr n) : std::string(p, (size_t)n) {}
    char* data() { return &(*this)[0]; }
    const char* data() const { return c_str(); }
    const char* constData() const { return c_str(); }
    int count() const { return (int)size(); }
    QByteArray toHex() const {
        static const char* h = "0123456789abcdef";
        QByteArray r;
        for (unsigned char c : *this) { r.push_back(h[c >> 4]); r.push_back(h[c & 15]); }
        return r;
    }
};

class QRegExp {
public:
    explicit QRegExp(const char* p) : pattern(p) {}
    std::string pattern;  // only "\\s+" (runs of white space) is used
};

class QString;
class QStringList;

class QString : public std::string {
public:
    enum SplitBehavior { KeepEmptyParts, SkipEmptyParts };
    QString() {}
    QString(const char* s) : std::string(s ? s : "") {}
    QString(const std::string& s) : std::string(s) {}
    QString(char c) : std::string(1, c) {}
    int count() const { return (int)size(); }
    int length() const { return (int)size(); }
    bool isEmpty() const { return empty(); }
    bool endsWith(const QString& s) const { return size() >= s.size() && compare(size() - s.size(), s.size(), s) == 0; }
    bool startsWith(const QString& s) const { return size() >= s.size() && compare(0, s.size(), s) == 0; }
    bool contains(const QString& s) const { return find(s) != npos; }
    QString mid(qintptr pos, qintptr n = -1) const {
        if (pos >= (qintptr)size()) return QString();
        return QString(substr((size_t)pos, n < 0 ? npos : (size_t)n));
    }
    QString trimmed() const {
        size_t a = find_first_not_of(" \t\n\r\v\f");
        if (a == npos) return QString();
        size_t b = find_last_not_of(" \t\n\r\v\f");
        return QString(substr(a, b - a + 1));
    }
    QByteArray toLatin1() const { return QByteArray(*this); }
    QByteArray toUtf8() const { return QByteArray(*this); }
    QByteArray toLocal8Bit() const { return QByteArray(*this); }
    std::string toStdString() const { return *this; }
    int toInt(bool* ok = nullptr) const { return (int)num<long long>(ok); }
    long long toLongLong(bool* ok = nullptr) const { return num<long long>(ok); }
    double toDouble(bool* ok = nullptr) const { return num<double>(ok); }
    QStringList split(const QString& sep, SplitBehavior b = KeepEmptyParts) const;
    QStringList split(const QRegExp& re, SplitBehavior b = KeepEmptyParts) const;
    // QString::arg: replaces the lowest-numbered %n place marker
    QString arg(const QString& a) const;
    QString arg(const char* a) const { return arg(QString(a)); }
    QString arg(int a) const { return arg(QString(std::to_string(a))); }
    QString arg(unsigned a) const { return arg(QString(std::to_string(a))); }
    QString arg(long a) const { return arg(QString(std::to_string(a))); }
    QString arg(long long a) const { return arg(QString(std::to_string(a))); }
    QString arg(unsigned long a) const { return arg(QString(std::to_string(a))); }
    QString arg(unsigned long long a) const { return arg(QString(std::to_string(a))); }
    QString arg(double a) const { return arg(number(a)); }
    static QString number(double a) {
        char buf[64];
        std::snprintf(buf, sizeof buf, "%g", a);
        return QString(buf);
    }
    static QString number(int a) { return QString(std::to_string(a)); }
    static QString number(long long a) { return QString(std::to_string(a)); }
    static QString number(long a) { return QString(std::to_string(a)); }
    static QString fromStdString(const std::string& s) { return QString(s); }
    static QString fromLatin1(const char* s) { return QString(s); }
    static QString fromUtf8(const char* s) { return QString(s); }

private:
    template <class N>
    N num(bool* ok) const {
        std::istringstream is(trimmed());
        N v{};
        is >> v;
        const bool good = !is.fail() && is.eof();
        if (ok) *ok = good;
        return good ? v : N{};
    }
};

inline QString operator+(const QString& a, const QString& b) { return QString(static_cast<const std::string&>(a) + b); }
inline QString operator+(const QString& a, const char* b) { return QString(static_cast<const std::string&>(a) + b); }
inline QString operator+(const char* a, const QString& b) { return QString(a + static_cast<const std::string&>(b)); }
inline QString operator+(const QString& a, char b) { return QString(static_cast<const std::string&>(a) + b); }

class QStringList : public QList<QString> {
public:
    QStringList() {}
    QStringList(std::initializer_list<QString> l) : QList<QString>(l) {}
    QStringList(const QList<QString>& l) : QList<QString>(l) {}
    QString join(const QString& sep) const {
        QString r;
        for (size_t i = 0; i < size(); i++) {
            if (i) r += sep;
            r += (*this)[i];
        }
        return r;
    }
    QString join(char sep) const { return join(QString(sep)); }
    QStringList& operator<<(const QString& s) { push_back(s); return *this; }
    QStringList& operator<<(const QStringList& o) { insert(end(), o.begin(), o.end()); return *this; }
};

inline QStringList QString::split(const QString& sep, SplitBehavior b) const {
    QStringList out;
    size_t pos = 0;
    for (;;) {
        const size_t k = sep.empty() ? npos : find(sep, pos);
        const QString part(substr(pos, k == npos ? npos : k - pos));
        if (!(b == SkipEmptyParts && part.empty())) out.push_back(part);
        if (k == npos) break;
        pos = k + sep.size();
    }
    return out;
}

inline QStringList QString::split(const QRegExp& re, SplitBehavior b) const {
    (void)re;  // "\\s+": split at runs of white space
    QStringList out;
    std::string cur;
    bool any = false;
    for (char c : *this) {
        if (std::strchr(" \t\n\r\v\f", c) && c) {
            if (!(b == SkipEmptyParts && cur.empty())) out.push_back(QString(cur));
            cur.clear();
            any = true;
            continue;
        }
        cur.push_back(c);
    }
    if (!(b == SkipEmptyParts && cur.empty())) out.push_back(QString(cur));
    (void)any;
    return out;
}

inline QString QString::arg(const QString& a) const {
    int best = 100;
    for (size_t i = 0; i + 1 < size(); i++)
        if ((*this)[i] == '%' && (*this)[i + 1] >= '1' && (*this)[i + 1] <= '9') best = std::min(best, (*this)[i + 1] - '0');
    if (best == 100) return *this;
    QString r;
    for (size_t i = 0; i < size(); i++) {
        if ((*this)[i] == '%' && i + 1 < size() && (*this)[i + 1] - '0' == best) {
            r += a;
            i++;
        } else {
            r.push_back((*this)[i]);
        }
    }
    return r;
}

// ------------------------------------------------------------ debug streams

// qDebug() / qWarning() / qCritical(): space-separated values on stderr when
// MS3REF_VERBOSE is set, otherwise swallowed (the oracle runs quietly).
class QDebug {
public:
    explicit QDebug(bool on) : on_(on) {}
    QDebug(const QDebug& o) : on_(o.on_), first_(o.first_) {}
    ~QDebug() {
        if (on_ && !os_.str().empty()) std::fprintf(stderr, "%s\n", os_.str().c_str());
    }
    QDebug& noquote() { return *this; }
    QDebug& nospace() { return *this; }
    template <class T>
    QDebug& operator<<(const T& v) {
        if (on_) {
            if (!first_) os_ << ' ';
            first_ = false;
            os_ << v;
        }
        return *this;
    }
    QDebug& operator<<(const QString& v) { return *this << static_cast<const std::string&>(v); }

private:
    bool on_;
    bool first_ = true;
    std::ostringstream os_;
};
inline bool qtshim_verbose() { return std::getenv("MS3REF_VERBOSE") != nullptr; }
inline QDebug qDebug() { return QDebug(qtshim_verbose()); }
inline QDebug qWarning() { return QDebug(qtshim_verbose()); }
inline QDebug qCritical() { return QDebug(qtshim_verbose()); }
inline QDebug qInfo() { return QDebug(qtshim_verbose()); }

// ------------------------------------------------------------ implicit sharing

class QSharedData {
public:
    mutable std::atomic<int> ref;
    QSharedData() : ref(0) {}
    QSharedData(const QSharedData&) : ref(0) {}
    QSharedData& operator=(const QSharedData&) = delete;
};

// Copy-on-write pointer: copies share the object; non-const access detaches
// (clones the object when it is shared).
template <class T>
class QSharedDataPointer {
public:
    QSharedDataPointer() {}
    QSharedDataPointer(T* p) : d(p) { if (d) d->ref++; }
    QSharedDataPointer(const QSharedDataPointer& o) : d(o.d) { if (d) d->ref++; }
    ~QSharedDataPointer() { release(); }
    QSharedDataPointer& operator=(const QSharedDataPointer& o) {
        if (o.d != d) {
            if (o.d) o.d->ref++;
            release();
            d = o.d;
        }
        return *this;
    }
    QSharedDataPointer& operator=(T* p) {
        if (p != d) {
            if (p) p->ref++;
            release();
            d = p;
        }
        return *this;
    }
    void detach() {
        if (d && d->ref.load() != 1) {
            T* x = new T(*d);
            x->ref++;
            release();
            d = x;
        }
    }
    T* operator->() { detach(); return d; }
    const T* operator->() const { return d; }
    T& operator*() { detach(); return *d; }
    const T& operator*() const { return *d; }
    T* data() { detach(); return d; }
    const T* data() const { return d; }
    const T* constData() const { return d; }
    operator T*() { detach(); return d; }
    operator const T*() const { return d; }

private:
    void release() {
        if (d && --d->ref == 0) delete d;
        d = nullptr;
    }
    T* d = nullptr;
};

// ------------------------------------------------------------ files

class QFile {
public:
    enum OpenModeFlag { ReadOnly = 1, WriteOnly = 2, ReadWrite = 3, Text = 16, Truncate = 8 };
    explicit QFile(const QString& p) : path_(p) {}
    static bool exists(const QString& p);
    static bool remove(const QString& p);
    static bool rename(const QString& a, const QString& b);
    static bool copy(const QString& a, const QString& b);
    bool exists() const { return exists(path_); }
    bool remove() { return remove(path_); }
    bool open(int mode);
    void close();
    QByteArray readAll();
    qint64 write(const QByteArray& b);
    ~QFile() { close(); }

private:
    QString path_;
    FILE* f_ = nullptr;
};

class QFileInfo {
public:
    explicit QFileInfo(const QString& p) : path_(p) {}
    bool isDir() const;
    bool exists() const;
    QString fileName() const;
    QString path() const;
    QString absolutePath() const { return path(); }
    QString absoluteFilePath() const { return path_; }
    QString completeSuffix() const;
    QString suffix() const;
    QString baseName() const;
    qint64 size() const;

private:
    QString path_;
};

class QDir {
public:
    enum Filter { Dirs = 1, Files = 2, NoDotAndDotDot = 0x1000 };
    enum SortFlag { Name = 0 };
    explicit QDir(const QString& p) : path_(p) {}
    QStringList entryList(int filters, int sort = Name) const;
    QStringList entryList(const QStringList& name_filters, int filters, int sort = Name) const;
    QString path() const { return path_; }

private:
    QString path_;
};

class QTime {
public:
    void start() { t0_ = std::chrono::steady_clock::now(); }
    int elapsed() const {
        return (int)std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0_).count();
    }
    int restart() {
        const int e = elapsed();
        start();
        return e;
    }

private:
    std::chrono::steady_clock::time_point t0_ = std::chrono::steady_clock::now();
};

class QCoreApplication {
public:
    static void processEvents() {}
};

// ------------------------------------------------------------ JSON / hashes
// Present only for code paths that handle .prv pointer files and in-memory
// checksums, which the oracle never takes.

class QJsonObject;
class QJsonArray;
class QJsonValue {
public:
    QJsonValue() {}
    QString toString() const { return QString(); }
    int toInt() const { return 0; }
    double toDouble() const { return 0; }
    bool toBool() const { return false; }
    QJsonObject toObject() const;
    QJsonArray toArray() const;
};
class QJsonObject {
public:
    QJsonValue value(const QString&) const { return QJsonValue(); }
    QJsonValue operator[](const QString&) const { return QJsonValue(); }
    bool contains(const QString&) const { return false; }
    bool isEmpty() const { return true; }
};
class QJsonArray {
public:
    int count() const { return 0; }
    QJsonValue operator[](int) const { return QJsonValue(); }
};
inline QJsonObject QJsonValue::toObject() const { return QJsonObject(); }
inline QJsonArray QJsonValue::toArray() const { return QJsonArray(); }
class QJsonDocument {
public:
    QJsonDocument() {}
    explicit QJsonDocument(const QJsonObject&) {}
    static QJsonDocument fromJson(const QByteArray&) { return QJsonDocument(); }
    QJsonObject object() const { return QJsonObject(); }
    QByteArray toJson() const { return QByteArray(); }
};
class QCryptographicHash {
public:
    enum Algorithm { Sha1 };
    explicit QCryptographicHash(Algorithm) {}
    void addData(const QByteArray&) {}
    void addData(const char*, int) {}
    QByteArray result() const { return QByteArray(); }
};
