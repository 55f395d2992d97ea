// libcntr's plain-text herm_matrix format (print_to_file / read_from_file,
// cntr_herm_matrix_impl.hpp:1308-1560) on host buffers in libcntr's layout.  The format is the
// reference's, so that files move between the two codes; the writer formats numbers the way
// std::ostream does at a given precision (the %g conversion), the reader accepts any
// whitespace between tokens, as stream extraction does.
#include <cerrno>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nessi_io.h"

namespace {

using cplx = std::complex<double>;
thread_local std::string g_err;

int fail(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return 1;
}

long tri(long n) { return n * (n + 1) / 2; }  // elements of rows 0..n-1 of a packed triangle

// Buffered writer.
struct Out {
    FILE *f = nullptr;
    std::string buf;
    int prec = 16;
    bool ok = true;
    void flush() {
        if (!buf.empty() && fwrite(buf.data(), 1, buf.size(), f) != buf.size()) ok = false;
        buf.clear();
    }
    void put(const char *s) {
        buf += s;
        if (buf.size() > (1u << 20)) flush();
    }
    void num(double x) {
        char t[64];
        snprintf(t, sizeof t, " %.*g", prec, x);
        put(t);
    }
    void entry(const char *label, const int *idx, int nidx, const cplx *e, int es) {
        char t[64];
        put(label);
        for (int i = 0; i < nidx; i++) {
            snprintf(t, sizeof t, " %d", idx[i]);
            put(t);
        }
        for (int l = 0; l < es; l++) {
            num(e[l].real());
            num(e[l].imag());
        }
        put("\n");
    }
};

// Whitespace-separated tokens of a file, read in chunks.
struct In {
    FILE *f = nullptr;
    std::vector<char> buf = std::vector<char>(1 << 20);
    size_t pos = 0, len = 0;
    bool eof = false;
    int fill() {
        if (eof) return 0;
        len = fread(buf.data(), 1, buf.size(), f);
        pos = 0;
        if (len == 0) eof = true;
        return (int)len;
    }
    bool token(std::string &t) {
        t.clear();
        for (;;) {
            if (pos == len && !fill()) return !t.empty();
            char c = buf[pos];
            if (c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\f' || c == '\v') {
                pos++;
                if (!t.empty()) return true;
            } else {
                t.push_back(c);
                pos++;
            }
        }
    }
    bool skip(int n) {
        std::string t;
        for (int i = 0; i < n; i++)
            if (!token(t)) return false;
        return true;
    }
    bool real(double &x) {
        std::string t;
        if (!token(t)) return false;
        char *end = nullptr;
        errno = 0;
        x = strtod(t.c_str(), &end);
        return end && *end == '\0' && end != t.c_str();
    }
    bool integer(int &x) {
        std::string t;
        if (!token(t)) return false;
        char *end = nullptr;
        long v = strtol(t.c_str(), &end, 10);
        x = (int)v;
        return end && *end == '\0' && end != t.c_str();
    }
    // one element (label and indices skipped): es complex numbers into e (may be null to discard)
    bool element(int nlabel, cplx *e, int es) {
        if (!skip(nlabel)) return false;
        for (int l = 0; l < es; l++) {
            double re, im;
            if (!real(re) || !real(im)) return false;
            if (e) e[l] = cplx(re, im);
        }
        return true;
    }
};

struct Header {
    int nt, ntau, size1, sig;
};

int read_header(In &in, const char *file, Header &h) {
    std::string hash;
    if (!in.token(hash) || !in.integer(h.nt) || !in.integer(h.ntau) || !in.integer(h.size1) || !in.integer(h.sig))
        return fail("read G from file %s error in file", file);
    if (h.nt < -1 || h.ntau < 0 || h.size1 < 1 || (h.sig != 1 && h.sig != -1))
        return fail("read G from file %s error in file (header %d %d %d %d)", file, h.nt, h.ntau, h.size1, h.sig);
    return 0;
}

// The body of read_from_file / read_from_file(nt1): mat, then the rows / columns of the file's
// n time steps, kept where the time index is <= keep (keep = n reads all).
int read_body(In &in, const char *file, const Header &h, int keep, cplx *ret, cplx *les, cplx *tv, cplx *mat) {
    const int es = h.size1 * h.size1, M = h.ntau + 1;
    for (int j = 0; j <= h.ntau; j++)
        if (!in.element(2, mat + (long)j * es, es)) return fail("read G from file %s error at mat (%d)", file, j);
    if (h.nt < 0) return 0;
    for (int i = 0; i <= h.nt; i++)
        for (int j = 0; j <= i; j++)
            if (!in.element(3, i <= keep ? ret + (tri(i) + j) * es : nullptr, es))
                return fail("read G from file %s error at ret (%d,%d)", file, i, j);
    for (int i = 0; i <= h.nt; i++)
        for (int j = 0; j <= h.ntau; j++)
            if (!in.element(3, i <= keep ? tv + ((long)i * M + j) * es : nullptr, es))
                return fail("read G from file %s error at tv (%d,%d)", file, i, j);
    for (int j = 0; j <= h.nt; j++)
        for (int i = 0; i <= j; i++)
            if (!in.element(3, j <= keep ? les + (tri(j) + i) * es : nullptr, es))
                return fail("read G from file %s error at les (%d,%d)", file, i, j);
    return 0;
}

struct File {
    FILE *f;
    explicit File(FILE *x) : f(x) {}
    ~File() {
        if (f) fclose(f);
    }
};

}  // namespace

extern "C" {

const char *nessi_io_last_error(void) { return g_err.c_str(); }

int nessi_hm_print_to_file(const char *file, int nt, int ntau, int size1, int sig, const void *ret_,
                           const void *les_, const void *tv_, const void *mat_, int precision) {
    if (!file) return fail("print_to_file: null file name");
    if (nt < -1 || ntau < 0 || size1 < 1 || (sig != 1 && sig != -1))
        return fail("print_to_file: bad dimensions nt=%d ntau=%d size1=%d sig=%d", nt, ntau, size1, sig);
    if (!mat_ || (nt >= 0 && (!ret_ || !les_ || !tv_))) return fail("print_to_file: null component");
    if (precision < 0 || precision > 40) return fail("print_to_file: precision %d out of range", precision);
    const cplx *ret = (const cplx *)ret_, *les = (const cplx *)les_, *tv = (const cplx *)tv_,
               *mat = (const cplx *)mat_;
    File fh(fopen(file, "w"));
    if (!fh.f) return fail("print_to_file: cannot open %s: %s", file, strerror(errno));
    Out o;
    o.f = fh.f;
    o.prec = precision;
    const int es = size1 * size1, M = ntau + 1;
    char t[128];
    snprintf(t, sizeof t, "# %d %d %d  %d\n", nt, ntau, size1, sig);
    o.put(t);
    for (int j = 0; j <= ntau; j++) o.entry("mat:", &j, 1, mat + (long)j * es, es);
    o.put("\n");
    if (nt >= 0) {
        for (int i = 0; i <= nt; i++) {
            for (int j = 0; j <= i; j++) {
                const int ij[2] = {i, j};
                o.entry("ret:", ij, 2, ret + (tri(i) + j) * es, es);
            }
            o.put("\n");
        }
        o.put("\n");
        for (int i = 0; i <= nt; i++) {
            for (int j = 0; j <= ntau; j++) {
                const int ij[2] = {i, j};
                o.entry("tv:", ij, 2, tv + ((long)i * M + j) * es, es);
            }
            o.put("\n");
        }
        o.put("\n");
        for (int j = 0; j <= nt; j++) {
            for (int i = 0; i <= j; i++) {
                const int ij[2] = {i, j};
                o.entry("les:", ij, 2, les + (tri(j) + i) * es, es);
            }
            o.put("\n");
        }
        o.put("\n");
    }
    o.flush();
    if (!o.ok) return fail("print_to_file: write to %s failed", file);
    return 0;
}

int nessi_hm_file_header(const char *file, int *nt, int *ntau, int *size1, int *sig) {
    if (!file) return fail("read_from_file: null file name");
    File fh(fopen(file, "r"));
    if (!fh.f) return fail("read G from file %s: cannot open: %s", file, strerror(errno));
    In in;
    in.f = fh.f;
    Header h;
    if (read_header(in, file, h)) return 1;
    if (nt) *nt = h.nt;
    if (ntau) *ntau = h.ntau;
    if (size1) *size1 = h.size1;
    if (sig) *sig = h.sig;
    return 0;
}

int nessi_hm_read_from_file(const char *file, int nt, int ntau, int size1, int *sig, void *ret, void *les,
                            void *tv, void *mat) {
    if (!file) return fail("read_from_file: null file name");
    File fh(fopen(file, "r"));
    if (!fh.f) return fail("read G from file %s: cannot open: %s", file, strerror(errno));
    In in;
    in.f = fh.f;
    Header h;
    if (read_header(in, file, h)) return 1;
    if (h.nt > nt || h.ntau != ntau || h.size1 != size1)
        return fail("read G from file %s: file holds nt=%d ntau=%d size1=%d, buffers nt=%d ntau=%d size1=%d", file,
                    h.nt, h.ntau, h.size1, nt, ntau, size1);
    if (!mat || (h.nt >= 0 && (!ret || !les || !tv))) return fail("read_from_file: null component");
    if (read_body(in, file, h, h.nt, (cplx *)ret, (cplx *)les, (cplx *)tv, (cplx *)mat)) return 1;
    if (sig) *sig = h.sig;
    return 0;
}

int nessi_hm_read_from_file_nt1(const char *file, int nt1, int nt, int ntau, int size1, void *ret, void *les,
                                void *tv, void *mat) {
    if (!file) return fail("read_from_file: null file name");
    File fh(fopen(file, "r"));
    if (!fh.f) return fail("read G from file %s: cannot open: %s", file, strerror(errno));
    In in;
    in.f = fh.f;
    Header h;
    if (read_header(in, file, h)) return 1;
    if (nt1 < -1 || nt1 > nt) return fail("read_from_file: nt1 = %d > nt = %d", nt1, nt);
    if (nt1 > h.nt) return fail("read_from_file: nt1 = %d > nt = %d of %s", nt1, h.nt, file);
    if (h.ntau != ntau) return fail("read_from_file: ntau %d of %s /= %d", h.ntau, file, ntau);
    if (h.size1 != size1) return fail("read_from_file: size1 %d of %s /= %d", h.size1, file, size1);
    if (!mat || (nt1 >= 0 && (!ret || !les || !tv))) return fail("read_from_file: null component");
    return read_body(in, file, h, nt1, (cplx *)ret, (cplx *)les, (cplx *)tv, (cplx *)mat);
}

}  // extern "C"
