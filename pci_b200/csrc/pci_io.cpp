// Readers and writers of pconf's file formats (include/pci_io.h): the CSR
// stream pCONF.HIJ/JJJ, CONF.XIJ, CONF.RES, CONF.DET, CONF.GNT and CONF.INT.
// Plain host C++ with stdio; no CUDA.
#include <algorithm>
#include <cinttypes>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pci_gpu.h"
#include "../../include/pci_io.h"

namespace {

int fail(char *errbuf, int32_t errlen, const char *fmt, ...)
{
    if (errbuf && errlen > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(errbuf, (size_t)errlen, fmt, ap);
        va_end(ap);
    }
    return PCI_E_INPUT;
}

struct File {
    FILE *f = nullptr;
    explicit File(const char *path, const char *mode) { f = path ? fopen(path, mode) : nullptr; }
    ~File() { if (f) fclose(f); }
    bool ok() const { return f != nullptr; }
};

// gfortran subrecord limit: the longest subrecord payload of a sequential
// unformatted record with 4-byte markers.
constexpr int64_t SUBREC_MAX = 2147483639LL;

// One sequential record assembled from pieces and written with markers.
struct RecWriter {
    std::vector<std::pair<const void *, size_t>> parts;
    void add(const void *p, size_t n) { parts.push_back({p, n}); }
    bool write(FILE *f) const
    {
        int64_t total = 0;
        for (auto &p : parts) total += (int64_t)p.second;
        // split into subrecords; payload streamed across the parts
        size_t pi = 0, po = 0;
        int64_t left = total;
        bool first = true;
        do {
            const int64_t n = std::min(left, SUBREC_MAX);
            const bool more = left > n;
            int32_t head = more ? -(int32_t)n : (int32_t)n;
            int32_t tail = first ? (int32_t)n : -(int32_t)n;
            if (fwrite(&head, 4, 1, f) != 1) return false;
            int64_t todo = n;
            while (todo > 0) {
                const size_t avail = parts[pi].second - po;
                const size_t take = (size_t)std::min<int64_t>(todo, (int64_t)avail);
                if (take && fwrite((const char *)parts[pi].first + po, 1, take, f) != take) return false;
                po += take;
                todo -= (int64_t)take;
                if (po == parts[pi].second) { pi++; po = 0; }
            }
            if (fwrite(&tail, 4, 1, f) != 1) return false;
            left -= n;
            first = false;
        } while (left > 0);
        return true;
    }
};

// Read one whole sequential record (all subrecords) into buf.
bool read_record(FILE *f, std::vector<char> &buf)
{
    buf.clear();
    while (true) {
        int32_t head;
        if (fread(&head, 4, 1, f) != 1) return false;
        const int64_t n = head < 0 ? -(int64_t)head : (int64_t)head;
        const size_t at = buf.size();
        buf.resize(at + (size_t)n);
        if (n && fread(buf.data() + at, 1, (size_t)n, f) != (size_t)n) return false;
        int32_t tail;
        if (fread(&tail, 4, 1, f) != 1) return false;
        if ((tail < 0 ? -(int64_t)tail : (int64_t)tail) != n) return false;
        if (head >= 0) return true;
    }
}

// Skip one sequential record, returning its payload length.
bool skip_record(FILE *f, int64_t *len)
{
    int64_t total = 0;
    while (true) {
        int32_t head;
        if (fread(&head, 4, 1, f) != 1) return false;
        const int64_t n = head < 0 ? -(int64_t)head : (int64_t)head;
        if (fseeko(f, (off_t)n, SEEK_CUR) != 0) return false;
        int32_t tail;
        if (fread(&tail, 4, 1, f) != 1) return false;
        if ((tail < 0 ? -(int64_t)tail : (int64_t)tail) != n) return false;
        total += n;
        if (head >= 0) break;
    }
    if (len) *len = total;
    return true;
}

template <typename T>
T get(const std::vector<char> &b, size_t off)
{
    T v;
    memcpy(&v, b.data() + off, sizeof(T));
    return v;
}

// Fortran Fw.d: right-justified fixed notation, asterisks when it does not fit.
std::string fmt_f(double x, int w, int d)
{
    char tmp[128];
    snprintf(tmp, sizeof tmp, "%*.*f", w, d, x);
    std::string s(tmp);
    if ((int)s.size() > w) return std::string((size_t)w, '*');
    return s;
}

std::string fmt_i(long long x, int w)
{
    char tmp[64];
    snprintf(tmp, sizeof tmp, "%*lld", w, x);
    std::string s(tmp);
    if ((int)s.size() > w) return std::string((size_t)w, '*');
    return s;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------ CSR stream ---

int pci_io_write_csr(const char *path, int64_t nd, int64_t nnz, const int64_t *rowptr, const int32_t *col,
                     const void *val, int32_t val_bytes, char *errbuf, int32_t errlen)
{
    if (nd < 0 || nnz < 0 || !rowptr || (nnz && (!col || !val)))
        return fail(errbuf, errlen, "write_csr: bad arguments");
    if (val_bytes != 8 && val_bytes != 4) return fail(errbuf, errlen, "write_csr: val_bytes must be 8 or 4");
    if (rowptr[0] != 0 || rowptr[nd] != nnz) return fail(errbuf, errlen, "write_csr: rowptr must run from 0 to nnz");
    File F(path, "wb");
    if (!F.ok()) return fail(errbuf, errlen, "write_csr: cannot open %s", path ? path : "(null)");
    bool ok = fwrite(&nd, 8, 1, F.f) == 1 && fwrite(&nnz, 8, 1, F.f) == 1 &&
              fwrite(rowptr, 8, (size_t)nd + 1, F.f) == (size_t)nd + 1 &&
              fwrite(col, 4, (size_t)nnz, F.f) == (size_t)nnz &&
              fwrite(val, (size_t)val_bytes, (size_t)nnz, F.f) == (size_t)nnz;
    if (!ok) return fail(errbuf, errlen, "write_csr: write to %s failed", path);
    return PCI_OK;
}

int pci_io_read_csr_header(const char *path, int64_t *nd, int64_t *nnz, int32_t *val_bytes, char *errbuf,
                           int32_t errlen)
{
    File F(path, "rb");
    if (!F.ok()) return fail(errbuf, errlen, "read_csr: cannot open %s", path ? path : "(null)");
    int64_t h[2];
    if (fread(h, 8, 2, F.f) != 2) return fail(errbuf, errlen, "read_csr: %s is shorter than its header", path);
    if (h[0] < 0 || h[1] < 0) return fail(errbuf, errlen, "read_csr: negative Nd or nnz in %s", path);
    if (fseeko(F.f, 0, SEEK_END) != 0) return fail(errbuf, errlen, "read_csr: cannot seek %s", path);
    const int64_t size = (int64_t)ftello(F.f);
    const int64_t base = 16 + (h[0] + 1) * 8 + h[1] * 4;
    int32_t vb = 0;
    if (size == base + h[1] * 8) vb = 8;
    else if (size == base + h[1] * 4) vb = 4;
    else return fail(errbuf, errlen, "read_csr: size of %s (%" PRId64 " bytes) matches neither 8- nor 4-byte values",
                     path, size);
    if (h[1] == 0) vb = 8;
    if (nd) *nd = h[0];
    if (nnz) *nnz = h[1];
    if (val_bytes) *val_bytes = vb;
    return PCI_OK;
}

int pci_io_read_csr(const char *path, int64_t nd, int64_t nnz, int64_t *rowptr, int32_t *col, void *val,
                    int32_t val_bytes, char *errbuf, int32_t errlen)
{
    int64_t fnd, fnnz;
    int32_t fvb;
    int rc = pci_io_read_csr_header(path, &fnd, &fnnz, &fvb, errbuf, errlen);
    if (rc) return rc;
    if (fnd != nd) return fail(errbuf, errlen, "read_csr: file Nd (%" PRId64 ") /= Nd (%" PRId64 ")", fnd, nd);
    if (fnnz != nnz) return fail(errbuf, errlen, "read_csr: file nnz (%" PRId64 ") /= nnz (%" PRId64 ")", fnnz, nnz);
    if (fvb != val_bytes && nnz > 0) return fail(errbuf, errlen, "read_csr: file holds %d-byte values", fvb);
    if (!rowptr || (nnz && (!col || !val))) return fail(errbuf, errlen, "read_csr: null array");
    File F(path, "rb");
    if (!F.ok() || fseeko(F.f, 16, SEEK_SET) != 0) return fail(errbuf, errlen, "read_csr: cannot reopen %s", path);
    bool ok = fread(rowptr, 8, (size_t)nd + 1, F.f) == (size_t)nd + 1 &&
              fread(col, 4, (size_t)nnz, F.f) == (size_t)nnz &&
              fread(val, (size_t)val_bytes, (size_t)nnz, F.f) == (size_t)nnz;
    if (!ok) return fail(errbuf, errlen, "read_csr: %s ended early", path);
    if (rowptr[0] != 0 || rowptr[nd] != nnz) return fail(errbuf, errlen, "read_csr: rowptr does not run from 0 to nnz");
    for (int64_t i = 0; i < nd; i++)
        if (rowptr[i + 1] < rowptr[i]) return fail(errbuf, errlen, "read_csr: rowptr decreases at row %" PRId64, i + 1);
    return PCI_OK;
}

// ----------------------------------------------------- CONF.HIJ / CONF.JJJ ---

// Appends the records of rows row0+1 .. row0+n (1-based) of a CSR slice:
// (int32 row, int32 col, real64 value) per non-zero element.
static bool hij_records(FILE *f, int64_t row0, int64_t n, const int64_t *rowptr, const int32_t *col, const double *val,
                        int64_t *written)
{
    struct Rec {
        int32_t r, c;
        double v;
    };
    static_assert(sizeof(Rec) == 16, "record layout");
    std::vector<Rec> buf;
    buf.reserve(1 << 16);
    for (int64_t i = 0; i < n; i++) {
        for (int64_t l = rowptr[i] - rowptr[0]; l < rowptr[i + 1] - rowptr[0]; l++) {
            if (val[l] == 0.0) continue;   // sort.f90 drops exact zeros
            buf.push_back(Rec{(int32_t)(row0 + i + 1), col[l], val[l]});
            if (buf.size() == buf.capacity()) {
                if (fwrite(buf.data(), sizeof(Rec), buf.size(), f) != buf.size()) return false;
                *written += (int64_t)buf.size();
                buf.clear();
            }
        }
    }
    if (!buf.empty() && fwrite(buf.data(), sizeof(Rec), buf.size(), f) != buf.size()) return false;
    *written += (int64_t)buf.size();
    return true;
}

int pci_io_write_hij(const char *path, int64_t nd, const int64_t *rowptr, const int32_t *col, const double *val,
                     char *errbuf, int32_t errlen)
{
    if (nd < 0 || nd > INT32_MAX || !rowptr || (rowptr[nd] > rowptr[0] && (!col || !val)))
        return fail(errbuf, errlen, "write_hij: bad arguments (Nd must fit a 4-byte integer)");
    File F(path, "wb");
    if (!F.ok()) return fail(errbuf, errlen, "write_hij: cannot open %s", path ? path : "(null)");
    int64_t count = 0;
    if (fwrite(&count, 8, 1, F.f) != 1) return fail(errbuf, errlen, "write_hij: write to %s failed", path);
    if (!hij_records(F.f, 0, nd, rowptr, col, val, &count))
        return fail(errbuf, errlen, "write_hij: write to %s failed", path);
    if (fseeko(F.f, 0, SEEK_SET) != 0 || fwrite(&count, 8, 1, F.f) != 1)
        return fail(errbuf, errlen, "write_hij: cannot write the count of %s", path);
    return PCI_OK;
}

int pci_io_append_hij(const char *path, int64_t row0, int64_t nrows, const int64_t *rowptr, const int32_t *col,
                      const double *val, char *errbuf, int32_t errlen)
{
    if (row0 < 0 || nrows < 0 || row0 + nrows > INT32_MAX || !rowptr || (rowptr[nrows] > rowptr[0] && (!col || !val)))
        return fail(errbuf, errlen, "append_hij: bad arguments");
    File F(path, row0 == 0 ? "wb+" : "rb+");
    if (!F.ok()) return fail(errbuf, errlen, "append_hij: cannot open %s", path ? path : "(null)");
    int64_t count = 0;
    if (row0 == 0) {
        if (fwrite(&count, 8, 1, F.f) != 1) return fail(errbuf, errlen, "append_hij: write to %s failed", path);
    } else {
        if (fread(&count, 8, 1, F.f) != 1 || count < 0) return fail(errbuf, errlen, "append_hij: %s has no count", path);
        if (fseeko(F.f, 0, SEEK_END) != 0) return fail(errbuf, errlen, "append_hij: cannot seek %s", path);
        if ((int64_t)ftello(F.f) != 8 + 16 * count)
            return fail(errbuf, errlen, "append_hij: %s is not a complete record stream", path);
    }
    if (!hij_records(F.f, row0, nrows, rowptr, col, val, &count))
        return fail(errbuf, errlen, "append_hij: write to %s failed", path);
    if (fseeko(F.f, 0, SEEK_SET) != 0 || fwrite(&count, 8, 1, F.f) != 1)
        return fail(errbuf, errlen, "append_hij: cannot write the count of %s", path);
    return PCI_OK;
}

int pci_io_read_hij(const char *path, int64_t cap, int32_t *row, int32_t *col, double *val, int64_t *count,
                    char *errbuf, int32_t errlen)
{
    File F(path, "rb");
    if (!F.ok()) return fail(errbuf, errlen, "read_hij: cannot open %s", path ? path : "(null)");
    int64_t n = 0;
    if (fread(&n, 8, 1, F.f) != 1 || n < 0) return fail(errbuf, errlen, "read_hij: %s has no count", path);
    if (count) *count = n;
    if (cap <= 0) return PCI_OK;
    if (!row || !col || !val) return fail(errbuf, errlen, "read_hij: null array");
    const int64_t m = std::min(cap, n);
    for (int64_t i = 0; i < m; i++) {
        int32_t rc[2];
        double v;
        if (fread(rc, 4, 2, F.f) != 2 || fread(&v, 8, 1, F.f) != 1)
            return fail(errbuf, errlen, "read_hij: %s ended at record %" PRId64, path, i + 1);
        row[i] = rc[0];
        col[i] = rc[1];
        val[i] = v;
    }
    return PCI_OK;
}

// -------------------------------------------------------------- CONF.XIJ ---

int pci_io_write_xij(const char *path, int32_t nlv, int64_t nd, const double *Tk, const double *Tj, const double *X,
                     char *errbuf, int32_t errlen)
{
    if (nlv < 0 || nd < 0 || nd > INT32_MAX || (nlv && (!Tk || !Tj || (nd && !X))))
        return fail(errbuf, errlen, "write_xij: bad arguments (Nd must fit a 4-byte integer)");
    File F(path, "wb");
    if (!F.ok()) return fail(errbuf, errlen, "write_xij: cannot open %s", path ? path : "(null)");
    const int32_t nd4 = (int32_t)nd;
    for (int32_t n = 0; n < nlv; n++) {
        RecWriter r;
        r.add(&Tk[n], 8);
        r.add(&Tj[n], 8);
        r.add(&nd4, 4);
        r.add(X + (size_t)n * (size_t)nd, (size_t)nd * 8);
        if (!r.write(F.f)) return fail(errbuf, errlen, "write_xij: write to %s failed", path);
    }
    return PCI_OK;
}

int pci_io_read_xij(const char *path, int32_t nlv_max, int64_t nd, double *Tk, double *Tj, double *X,
                    int32_t *nread, char *errbuf, int32_t errlen)
{
    if (nread) *nread = 0;
    File F(path, "rb");
    if (!F.ok()) return fail(errbuf, errlen, "read_xij: cannot open %s", path ? path : "(null)");
    std::vector<char> b;
    int32_t n = 0;
    for (; n < nlv_max; n++) {
        if (!read_record(F.f, b)) {
            if (feof(F.f) && b.empty()) break;
            return fail(errbuf, errlen, "read_xij: record %d of %s is truncated", n + 1, path);
        }
        if (b.size() < 20) return fail(errbuf, errlen, "read_xij: record %d is too short", n + 1);
        const int32_t rnd = get<int32_t>(b, 16);
        if (rnd != nd) return fail(errbuf, errlen, "read_xij: record %d holds Nd = %d, expected %" PRId64, n + 1, rnd, nd);
        if ((int64_t)b.size() != 20 + 8 * nd)
            return fail(errbuf, errlen, "read_xij: record %d length %zu does not match Nd", n + 1, b.size());
        if (Tk) Tk[n] = get<double>(b, 0);
        if (Tj) Tj[n] = get<double>(b, 8);
        if (X) memcpy(X + (size_t)n * (size_t)nd, b.data() + 20, (size_t)nd * 8);
    }
    if (nread) *nread = n;
    return PCI_OK;
}

// -------------------------------------------------------------- CONF.RES ---

int pci_io_write_res(const char *path, int32_t append, int32_t kbrt, int32_t nc, int64_t nd, double gj, int32_t nlv,
                     const double *Tj, const double *Tk, double ecore, char *errbuf, int32_t errlen)
{
    static const char *label[3] = {"COULOMB", "GAUNT  ", "BREIT  "};
    if (kbrt < 0 || kbrt > 2 || nlv < 0 || (nlv && (!Tj || !Tk))) return fail(errbuf, errlen, "write_res: bad arguments");
    const double DPRy = 109737.315709;
    File F(path, append ? "a" : "w");
    if (!F.ok()) return fail(errbuf, errlen, "write_res: cannot open %s", path ? path : "(null)");
    std::string out;
    out += " " + std::string(80, '=') + "\n";
    out += "    Energy levels (" + std::string(label[kbrt]) + " Nc=" + fmt_i(nc, 7) + " Nd=" + fmt_i(nd, 9) +
           "); Gj =" + fmt_f(gj, 7, 4) + "\n";
    out += "    N" + std::string(6, ' ') + "JTOT" + std::string(12, ' ') + "EV" + std::string(16, ' ') + "ET" +
           std::string(9, ' ') + "DEL(CM**-1)\n";
    out += " " + std::string(80, '-') + "\n";
    std::vector<double> ev((size_t)nlv);
    for (int32_t j = 0; j < nlv; j++) {
        ev[(size_t)j] = Tk[j] + 4.0 * gj * Tj[j] * (Tj[j] + 1.0);
        const double dt = ev[(size_t)j] - ecore;
        const double del = (ev[0] - ev[(size_t)j]) * 2 * DPRy;
        out += "   " + fmt_i(j + 1, 3) + fmt_f(Tj[j], 14, 9) + fmt_f(ev[(size_t)j], 14, 8) + fmt_f(dt, 18, 6) +
               fmt_f(del, 15, 2) + "\n";
    }
    out += " " + std::string(80, '=') + "\n";
    if (fwrite(out.data(), 1, out.size(), F.f) != out.size()) return fail(errbuf, errlen, "write_res: write failed");
    return PCI_OK;
}

// -------------------------------------------------------------- CONF.DET ---

int pci_io_write_det(const char *path, int32_t ne, int64_t nd, int32_t nsu, const int32_t *Iarr, char *errbuf,
                     int32_t errlen)
{
    if (ne <= 0 || nd < 0 || nd > INT32_MAX || (nd && !Iarr)) return fail(errbuf, errlen, "write_det: bad arguments");
    File F(path, "wb");
    if (!F.ok()) return fail(errbuf, errlen, "write_det: cannot open %s", path ? path : "(null)");
    const int32_t h[2] = {(int32_t)nd, nsu};
    RecWriter r0;
    r0.add(h, 8);
    if (!r0.write(F.f)) return fail(errbuf, errlen, "write_det: write failed");
    for (int64_t i = 0; i < nd; i++) {
        RecWriter r;
        r.add(Iarr + (size_t)i * (size_t)ne, (size_t)ne * 4);
        if (!r.write(F.f)) return fail(errbuf, errlen, "write_det: write failed");
    }
    return PCI_OK;
}

int pci_io_read_det_header(const char *path, int64_t *nd, int32_t *nsu, int32_t *ne, char *errbuf, int32_t errlen)
{
    File F(path, "rb");
    if (!F.ok()) return fail(errbuf, errlen, "read_det: cannot open %s", path ? path : "(null)");
    std::vector<char> b;
    if (!read_record(F.f, b) || b.size() != 8) return fail(errbuf, errlen, "read_det: first record is not Nd, Nsu");
    if (nd) *nd = get<int32_t>(b, 0);
    if (nsu) *nsu = get<int32_t>(b, 4);
    if (ne) {
        int64_t len = 0;
        *ne = 0;
        if (get<int32_t>(b, 0) > 0) {
            if (!skip_record(F.f, &len) || len % 4) return fail(errbuf, errlen, "read_det: bad determinant record");
            *ne = (int32_t)(len / 4);
        }
    }
    return PCI_OK;
}

int pci_io_read_det(const char *path, int32_t ne, int64_t nd, int32_t *Iarr, char *errbuf, int32_t errlen)
{
    File F(path, "rb");
    if (!F.ok()) return fail(errbuf, errlen, "read_det: cannot open %s", path ? path : "(null)");
    std::vector<char> b;
    if (!read_record(F.f, b) || b.size() != 8) return fail(errbuf, errlen, "read_det: first record is not Nd, Nsu");
    if (get<int32_t>(b, 0) != nd) return fail(errbuf, errlen, "read_det: file Nd (%d) /= Nd", get<int32_t>(b, 0));
    for (int64_t i = 0; i < nd; i++) {
        // Rdet: a short file is a premature end at determinant i
        if (!read_record(F.f, b) || (int64_t)b.size() != 4LL * ne)
            return fail(errbuf, errlen, "Rdet: premature end of file in %s at idet=%" PRId64, path, i + 1);
        memcpy(Iarr + (size_t)i * (size_t)ne, b.data(), (size_t)ne * 4);
    }
    return PCI_OK;
}

// -------------------------------------------------------------- CONF.GNT ---

int pci_io_write_gnt(const char *path, int32_t nlx, int32_t ngaunt, const int32_t *per_wave, const int32_t *In,
                     const double *Gnt, char *errbuf, int32_t errlen)
{
    if (nlx < 0 || ngaunt < 0 || !per_wave || (ngaunt && (!In || !Gnt)))
        return fail(errbuf, errlen, "write_gnt: bad arguments");
    File F(path, "wb");
    if (!F.ok()) return fail(errbuf, errlen, "write_gnt: cannot open %s", path ? path : "(null)");
    const int32_t h[2] = {nlx, ngaunt};
    RecWriter r0, r1, r2, r3;
    r0.add(h, 8);
    r1.add(per_wave, (size_t)(nlx + 1) * 4);
    r2.add(In, (size_t)ngaunt * 4);
    r3.add(Gnt, (size_t)ngaunt * 8);
    if (!(r0.write(F.f) && r1.write(F.f) && r2.write(F.f) && r3.write(F.f)))
        return fail(errbuf, errlen, "write_gnt: write failed");
    return PCI_OK;
}

int pci_io_read_gnt_header(const char *path, int32_t *nlx, int32_t *ngaunt, char *errbuf, int32_t errlen)
{
    File F(path, "rb");
    if (!F.ok()) return fail(errbuf, errlen, "read_gnt: cannot open %s", path ? path : "(null)");
    std::vector<char> b;
    if (!read_record(F.f, b)) return fail(errbuf, errlen, "read_gnt: no first record");
    // the reader falls back to a lone Ngaunt with Nlx = 5 (older files)
    if (b.size() == 8) {
        if (nlx) *nlx = get<int32_t>(b, 0);
        if (ngaunt) *ngaunt = get<int32_t>(b, 4);
    } else if (b.size() == 4) {
        if (nlx) *nlx = 5;
        if (ngaunt) *ngaunt = get<int32_t>(b, 0);
    } else {
        return fail(errbuf, errlen, "read_gnt: first record is neither (Nlx, Ngaunt) nor Ngaunt");
    }
    return PCI_OK;
}

int pci_io_read_gnt(const char *path, int32_t nlx, int32_t ngaunt, int32_t *per_wave, int32_t *In, double *Gnt,
                    char *errbuf, int32_t errlen)
{
    File F(path, "rb");
    if (!F.ok()) return fail(errbuf, errlen, "read_gnt: cannot open %s", path ? path : "(null)");
    std::vector<char> b;
    if (!read_record(F.f, b)) return fail(errbuf, errlen, "read_gnt: no first record");
    const bool old = b.size() == 4;
    if (!old && (b.size() != 8 || get<int32_t>(b, 0) != nlx || get<int32_t>(b, 4) != ngaunt))
        return fail(errbuf, errlen, "read_gnt: header does not match Nlx, Ngaunt");
    if (!old) {
        if (!read_record(F.f, b) || (int64_t)b.size() != 4LL * (nlx + 1))
            return fail(errbuf, errlen, "read_gnt: bad num_gaunts_per_partial_wave record");
        if (per_wave) memcpy(per_wave, b.data(), b.size());
    }
    if (!read_record(F.f, b) || (int64_t)b.size() != 4LL * ngaunt) return fail(errbuf, errlen, "read_gnt: bad In record");
    if (In) memcpy(In, b.data(), b.size());
    if (!read_record(F.f, b) || (int64_t)b.size() != 8LL * ngaunt) return fail(errbuf, errlen, "read_gnt: bad Gnt record");
    if (Gnt) memcpy(Gnt, b.data(), b.size());
    return PCI_OK;
}

int pci_io_gaunt_lut(int32_t ngaunt, const int32_t *In, const double *Gnt, double *lut, int64_t *nlut)
{
    if (ngaunt < 0 || (ngaunt && (!In || !Gnt))) return PCI_E_INPUT;
    int64_t mx = 0;
    for (int32_t i = 0; i < ngaunt; i++) {
        if (In[i] < 0) return PCI_E_INPUT;
        mx = std::max<int64_t>(mx, In[i]);
    }
    if (nlut) *nlut = mx + 1;
    if (lut) {
        std::fill(lut, lut + mx + 1, 0.0);
        for (int32_t i = 0; i < ngaunt; i++) lut[In[i]] = Gnt[i];
    }
    return PCI_OK;
}

// -------------------------------------------------------------- CONF.INT ---

int pci_io_read_int_header(const char *path, pci_int_header *hdr, char *errbuf, int32_t errlen)
{
    if (!hdr) return fail(errbuf, errlen, "read_int: null header");
    File F(path, "rb");
    if (!F.ok()) return fail(errbuf, errlen, "read_int: cannot open %s", path ? path : "(null)");
    std::vector<char> b;
    if (!read_record(F.f, b) || b.size() != 24) return fail(errbuf, errlen, "read_int: record 1 is not Ns,Nso,Nsp,Nsx,Ecore");
    hdr->ns = get<int32_t>(b, 0);
    hdr->nso = get<int32_t>(b, 4);
    hdr->nsp = get<int32_t>(b, 8);
    hdr->nsx = get<int32_t>(b, 12);
    hdr->ecore = get<double>(b, 16);
    if (!read_record(F.f, b) || (int64_t)b.size() != 16LL * hdr->nsx)
        return fail(errbuf, errlen, "read_int: record 2 is not (Nn,Kk,Ll,Jj) x Nsx");
    if (!skip_record(F.f, nullptr)) return fail(errbuf, errlen, "read_int: record 3 missing");
    if (!read_record(F.f, b) || b.size() != 8) return fail(errbuf, errlen, "read_int: record 4 is not Nhint,Kbrt");
    hdr->nhint = get<int32_t>(b, 0);
    hdr->kbrt = get<int32_t>(b, 4);
    int64_t len = 0;
    if (!skip_record(F.f, &len) || len != 8LL * hdr->nhint) return fail(errbuf, errlen, "read_int: bad Rint1 record");
    if (!skip_record(F.f, &len) || len != 4LL * hdr->nhint) return fail(errbuf, errlen, "read_int: bad Iint1 record");
    if (!read_record(F.f, b) || b.size() != 16) return fail(errbuf, errlen, "read_int: record 7 is not Ngint,Nlist,nrd");
    hdr->ngint = get<int64_t>(b, 0);
    hdr->nlist = get<int32_t>(b, 8);
    hdr->nrd = get<int32_t>(b, 12);
    if (!skip_record(F.f, &len)) return fail(errbuf, errlen, "read_int: Rint2 record missing");
    const int64_t per = hdr->ngint * (hdr->kbrt ? 2 : 1);
    if (per > 0 && len == 8 * per) hdr->r2_bytes = 8;
    else if (len == 4 * per) hdr->r2_bytes = 4;
    else return fail(errbuf, errlen, "read_int: Rint2 record length matches neither 4- nor 8-byte reals");
    return PCI_OK;
}

int pci_io_read_int(const char *path, const pci_int_header *hdr, int32_t *NnKkLlJj, double *Rint1, int32_t *Iint1,
                    void *Rint2, int32_t *Iint2, int32_t *Iint3, int64_t *IntOrd, char *errbuf, int32_t errlen)
{
    pci_int_header h;
    int rc = pci_io_read_int_header(path, &h, errbuf, errlen);
    if (rc) return rc;
    if (!hdr || h.nsx != hdr->nsx || h.nhint != hdr->nhint || h.ngint != hdr->ngint || h.nrd != hdr->nrd ||
        h.kbrt != hdr->kbrt || h.r2_bytes != hdr->r2_bytes)
        return fail(errbuf, errlen, "read_int: header does not match the file");
    File F(path, "rb");
    if (!F.ok()) return fail(errbuf, errlen, "read_int: cannot reopen %s", path);
    std::vector<char> b;
    auto take = [&](void *dst, int64_t bytes, const char *what) -> int {
        if (!read_record(F.f, b) || (int64_t)b.size() != bytes) return fail(errbuf, errlen, "read_int: bad %s record", what);
        if (dst && bytes) memcpy(dst, b.data(), (size_t)bytes);
        return PCI_OK;
    };
    if ((rc = take(nullptr, 24, "header"))) return rc;
    if ((rc = take(NnKkLlJj, 16LL * h.nsx, "orbital"))) return rc;
    if (!skip_record(F.f, nullptr)) return fail(errbuf, errlen, "read_int: record 3 missing");
    if ((rc = take(nullptr, 8, "Nhint"))) return rc;
    if ((rc = take(Rint1, 8LL * h.nhint, "Rint1"))) return rc;
    if ((rc = take(Iint1, 4LL * h.nhint, "Iint1"))) return rc;
    if ((rc = take(nullptr, 16, "Ngint"))) return rc;
    if ((rc = take(Rint2, (int64_t)h.r2_bytes * h.ngint * (h.kbrt ? 2 : 1), "Rint2"))) return rc;
    if ((rc = take(Iint2, 4 * h.ngint, "Iint2"))) return rc;
    if ((rc = take(Iint3, 4 * h.ngint, "Iint3"))) return rc;
    if ((rc = take(IntOrd, 8LL * h.nrd, "IntOrd"))) return rc;
    return PCI_OK;
}

int pci_io_write_int(const char *path, const pci_int_header *hdr, const int32_t *NnKkLlJj, const double *Rint1,
                     const int32_t *Iint1, const void *Rint2, const int32_t *Iint2, const int32_t *Iint3,
                     const int64_t *IntOrd, char *errbuf, int32_t errlen)
{
    if (!hdr || hdr->nsx < 0 || hdr->nhint < 0 || hdr->ngint < 0 || hdr->nrd < 0 ||
        (hdr->r2_bytes != 4 && hdr->r2_bytes != 8) || !NnKkLlJj || (hdr->nhint && (!Rint1 || !Iint1)) ||
        (hdr->ngint && (!Rint2 || !Iint2 || !Iint3)) || (hdr->nrd && !IntOrd))
        return fail(errbuf, errlen, "write_int: bad arguments");
    File F(path, "wb");
    if (!F.ok()) return fail(errbuf, errlen, "write_int: cannot open %s", path ? path : "(null)");
    const int32_t r1[4] = {hdr->ns, hdr->nso, hdr->nsp, hdr->nsx};
    const int32_t r4[2] = {hdr->nhint, hdr->kbrt};
    // record 3 (per-shell Nq, Nip) is not read by Rint; written empty
    RecWriter a, o, skip, n4, ri1, ii1, r7, ri2, ii2, ii3, io;
    a.add(r1, 16);
    a.add(&hdr->ecore, 8);
    o.add(NnKkLlJj, (size_t)hdr->nsx * 16);
    n4.add(r4, 8);
    ri1.add(Rint1, (size_t)hdr->nhint * 8);
    ii1.add(Iint1, (size_t)hdr->nhint * 4);
    r7.add(&hdr->ngint, 8);
    r7.add(&hdr->nlist, 4);
    r7.add(&hdr->nrd, 4);
    ri2.add(Rint2, (size_t)hdr->ngint * (hdr->kbrt ? 2 : 1) * (size_t)hdr->r2_bytes);
    ii2.add(Iint2, (size_t)hdr->ngint * 4);
    ii3.add(Iint3, (size_t)hdr->ngint * 4);
    io.add(IntOrd, (size_t)hdr->nrd * 8);
    for (const RecWriter *r : {&a, &o, &skip, &n4, &ri1, &ii1, &r7, &ri2, &ii2, &ii3, &io})
        if (!r->write(F.f)) return fail(errbuf, errlen, "write_int: write failed");
    return PCI_OK;
}

int pci_io_hint_lut(int32_t nhint, const double *Rint1, const int32_t *Iint1, int32_t nx, double *lut)
{
    if (nhint < 0 || nx <= 0 || !lut || (nhint && (!Rint1 || !Iint1))) return PCI_E_INPUT;
    const int64_t n = (int64_t)nx * nx;
    std::fill(lut, lut + n, 0.0);
    for (int32_t i = 0; i < nhint; i++) {
        if (Iint1[i] < 1 || Iint1[i] > n) return PCI_E_INPUT;
        lut[Iint1[i] - 1] = Rint1[i];
    }
    return PCI_OK;
}

}  // extern "C"
