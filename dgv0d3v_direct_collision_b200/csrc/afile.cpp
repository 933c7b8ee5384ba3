// afile.cpp -- the reference's on-disk A-arrays (WriteAarraysDGV,
// ReadAarraysDGV, ReadAarraysChnksDGV: readwrite.f90:1459-1484, 1066-1118,
// 1130-1243).
//
// A file is a Fortran unformatted sequential file of two records:
//   record 1: mm, nn                                   (int32, int32)
//   record 2: A_capphi(mm), A(nn), A_xi(nn), A_xi1(nn), A_phi(nn)
//             (int32, float64, int32, int32, int32; node indices 1-based)
// Records are framed the way gfortran writes them: a 4-byte signed length
// before and after the payload.  A record longer than a subrecord limit
// (2^31 - 9 bytes) is split into subrecords: a negative leading marker says
// that another subrecord follows, a negative trailing marker that this one
// continues an earlier one; the absolute values are the subrecord lengths.
// A chunked operator is a sequence of such files covering increasing ranges
// of basis nodes; reading adds their A_capphi arrays and concatenates the
// records in file order, as ReadAarraysChnksDGV does.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dgv_internal.h"

namespace dgv {

namespace {

constexpr long long kMaxSubrecord = 2147483639LL;  // 2^31 - 9

struct File {
    FILE *fp = nullptr;
    ~File()
    {
        if (fp) fclose(fp);
    }
};

// reads one (possibly split) record into buf; returns "" or an error message
std::string read_record(FILE *fp, std::vector<unsigned char> &buf)
{
    buf.clear();
    for (;;) {
        int32_t head = 0, tail = 0;
        if (fread(&head, 4, 1, fp) != 1) return "unexpected end of file at a record marker";
        const long long len = head < 0 ? -(long long)head : (long long)head;
        const size_t off = buf.size();
        buf.resize(off + (size_t)len);
        if (len && fread(buf.data() + off, 1, (size_t)len, fp) != (size_t)len) return "record shorter than its marker";
        if (fread(&tail, 4, 1, fp) != 1) return "unexpected end of file at a trailing marker";
        const long long tlen = tail < 0 ? -(long long)tail : (long long)tail;
        if (tlen != len) return "leading and trailing record markers disagree";
        if (head >= 0) return "";
    }
}

struct Piece {
    const void *p;
    size_t n;
};

// writes the concatenation of the pieces as one record, split into
// subrecords of at most maxsub bytes
bool write_record(FILE *fp, const std::vector<Piece> &pieces, long long maxsub)
{
    long long total = 0;
    for (const Piece &pc : pieces) total += (long long)pc.n;
    long long nsub = total == 0 ? 1 : (total + maxsub - 1) / maxsub;
    size_t ip = 0, ioff = 0;
    for (long long s = 0; s < nsub; s++) {
        const long long len = std::min(maxsub, total - s * maxsub);
        const int32_t head = (int32_t)(s + 1 < nsub ? -len : len);
        const int32_t tail = (int32_t)(s > 0 ? -len : len);
        if (fwrite(&head, 4, 1, fp) != 1) return false;
        long long left = len;
        while (left > 0) {
            const size_t take = (size_t)std::min<long long>(left, (long long)(pieces[ip].n - ioff));
            if (take && fwrite((const char *)pieces[ip].p + ioff, 1, take, fp) != take) return false;
            ioff += take;
            left -= (long long)take;
            if (ioff == pieces[ip].n) {
                ip++;
                ioff = 0;
            }
        }
        if (fwrite(&tail, 4, 1, fp) != 1) return false;
    }
    return true;
}

struct AArrays {
    std::vector<int32_t> capphi, xi, xi1, phi;
    std::vector<double> A;
};

// reads one file; returns "" or an error message
std::string read_one(const char *path, AArrays &out)
{
    File f;
    f.fp = fopen(path, "rb");
    if (!f.fp) return std::string("cannot open ") + path;
    std::vector<unsigned char> rec;
    std::string e = read_record(f.fp, rec);
    if (!e.empty()) return std::string(path) + ": " + e;
    if (rec.size() != 8) return std::string(path) + ": first record is not (mm, nn)";
    int32_t mm, nn;
    std::memcpy(&mm, rec.data(), 4);
    std::memcpy(&nn, rec.data() + 4, 4);
    if (mm < 0 || nn < 0) return std::string(path) + ": negative sizes";
    e = read_record(f.fp, rec);
    if (!e.empty()) return std::string(path) + ": " + e;
    if (rec.size() != 4 * (size_t)mm + 20 * (size_t)nn)
        return std::string(path) + ": second record has the wrong length for (mm, nn)";
    out.capphi.resize(mm);
    out.A.resize(nn);
    out.xi.resize(nn);
    out.xi1.resize(nn);
    out.phi.resize(nn);
    const unsigned char *p = rec.data();
    std::memcpy(out.capphi.data(), p, 4 * (size_t)mm);
    p += 4 * (size_t)mm;
    std::memcpy(out.A.data(), p, 8 * (size_t)nn);
    p += 8 * (size_t)nn;
    std::memcpy(out.xi.data(), p, 4 * (size_t)nn);
    p += 4 * (size_t)nn;
    std::memcpy(out.xi1.data(), p, 4 * (size_t)nn);
    p += 4 * (size_t)nn;
    std::memcpy(out.phi.data(), p, 4 * (size_t)nn);
    return "";
}

// reads and joins the files of a (chunked) operator; checks that every
// record's A_phi names the node whose records it is (1-based)
std::string read_all(const char *const *paths, int32_t nfiles, AArrays &all)
{
    if (!paths || nfiles < 1) return "need at least one path";
    for (int32_t i = 0; i < nfiles; i++) {
        if (!paths[i]) return "NULL path";
        AArrays part;
        std::string e = read_one(paths[i], part);
        if (!e.empty()) return e;
        if (i == 0) {
            all = std::move(part);
            continue;
        }
        if (part.capphi.size() != all.capphi.size()) return std::string(paths[i]) + ": A_capphi length differs";
        for (size_t k = 0; k < all.capphi.size(); k++) all.capphi[k] += part.capphi[k];
        all.A.insert(all.A.end(), part.A.begin(), part.A.end());
        all.xi.insert(all.xi.end(), part.xi.begin(), part.xi.end());
        all.xi1.insert(all.xi1.end(), part.xi1.begin(), part.xi1.end());
        all.phi.insert(all.phi.end(), part.phi.begin(), part.phi.end());
    }
    size_t k = 0;
    for (size_t node = 0; node < all.capphi.size(); node++) {
        if (all.capphi[node] < 0) return "negative A_capphi entry";
        for (int32_t r = 0; r < all.capphi[node]; r++, k++) {
            if (k >= all.phi.size()) return "sum(A_capphi) exceeds the record count";
            if (all.phi[k] != (int32_t)node + 1) return "A_phi does not match A_capphi (records out of node order)";
        }
    }
    if (k != all.phi.size()) return "sum(A_capphi) differs from the record count";
    return "";
}

std::string write_file(const char *path, int32_t N, int64_t nnz, const int32_t *capphi, const double *A,
                       const int32_t *xi, const int32_t *xi1, long long maxsub)
{
    if (nnz > INT32_MAX) return "more than 2^31-1 records (the format's sizes are int32)";
    std::vector<int32_t> phi((size_t)nnz);
    size_t k = 0;
    for (int32_t node = 0; node < N; node++)
        for (int32_t r = 0; r < capphi[node]; r++, k++) {
            if (k >= (size_t)nnz) return "sum(A_capphi) exceeds the record count";
            phi[k] = node + 1;
        }
    if (k != (size_t)nnz) return "sum(A_capphi) differs from the record count";
    File f;
    f.fp = fopen(path, "wb");
    if (!f.fp) return std::string("cannot create ") + path;
    const int32_t sizes[2] = {N, (int32_t)nnz};
    const bool ok = write_record(f.fp, {{sizes, 8}}, maxsub) &&
                    write_record(f.fp,
                                 {{capphi, 4 * (size_t)N},
                                  {A, 8 * (size_t)nnz},
                                  {xi, 4 * (size_t)nnz},
                                  {xi1, 4 * (size_t)nnz},
                                  {phi.data(), 4 * (size_t)nnz}},
                                 maxsub);
    if (!ok) return std::string("write failed for ") + path;
    return "";
}

thread_local std::string g_file_err;

}  // namespace

}  // namespace dgv

using namespace dgv;

extern "C" const char *dgv_file_error(void) { return g_file_err.c_str(); }

extern "C" int dgv_read_A_arrays(const char *const *paths, int32_t nfiles, int32_t N, int64_t *nnz_out,
                                 int32_t *capphi, double *A, int32_t *A_xi, int32_t *A_xi1)
{
    AArrays all;
    g_file_err = read_all(paths, nfiles, all);
    if (!g_file_err.empty()) return DGV_EINVAL;
    if ((long long)all.capphi.size() != (long long)N) {
        g_file_err = "A_capphi length differs from the node count N";
        return DGV_EINVAL;
    }
    if (nnz_out) *nnz_out = (int64_t)all.A.size();
    if (capphi) std::memcpy(capphi, all.capphi.data(), 4 * all.capphi.size());
    if (A) std::memcpy(A, all.A.data(), 8 * all.A.size());
    if (A_xi) std::memcpy(A_xi, all.xi.data(), 4 * all.xi.size());
    if (A_xi1) std::memcpy(A_xi1, all.xi1.data(), 4 * all.xi1.size());
    return DGV_OK;
}

extern "C" int dgv_write_A_arrays(const char *path, int32_t N, int64_t nnz, const int32_t *capphi, const double *A,
                                  const int32_t *A_xi, const int32_t *A_xi1, int64_t max_subrecord)
{
    if (!path || !capphi || N < 0 || nnz < 0 || (nnz > 0 && (!A || !A_xi || !A_xi1))) {
        g_file_err = "write_A_arrays: bad arguments";
        return DGV_EINVAL;
    }
    if (max_subrecord < 0 || max_subrecord > kMaxSubrecord) {
        g_file_err = "write_A_arrays: subrecord limit outside (0, 2^31-9]";
        return DGV_EINVAL;
    }
    g_file_err = write_file(path, N, nnz, capphi, A, A_xi, A_xi1, max_subrecord ? max_subrecord : kMaxSubrecord);
    return g_file_err.empty() ? DGV_OK : DGV_EINVAL;
}

extern "C" int dgv_read_A_files(dgv_ctx *ctx, const char *const *paths, int32_t nfiles)
{
    if (!ctx) return DGV_EINVAL;
    Ctx *c = &ctx->c;
    AArrays all;
    std::string e = read_all(paths, nfiles, all);
    if (!e.empty()) return set_err(c, DGV_EINVAL, "read_A_files: " + e);
    if ((long long)all.capphi.size() != c->grid.N)
        return set_err(c, DGV_EINVAL, "read_A_files: A_capphi length differs from the grid's node count");
    return dgv_load_A(ctx, (int64_t)all.A.size(), all.capphi.data(), all.A.data(), all.xi.data(), all.xi1.data(), 1);
}

extern "C" int dgv_write_A_file(dgv_ctx *ctx, const char *path, int64_t max_subrecord)
{
    if (!ctx) return DGV_EINVAL;
    Ctx *c = &ctx->c;
    if (!path) return set_err(c, DGV_EINVAL, "write_A_file: NULL path");
    if (max_subrecord < 0 || max_subrecord > kMaxSubrecord)
        return set_err(c, DGV_EINVAL, "write_A_file: subrecord limit outside (0, 2^31-9]");
    int64_t nnz = 0;
    int rc = dgv_export_A(ctx, &nnz, nullptr, nullptr, nullptr, nullptr);
    if (rc) return rc;
    std::vector<int32_t> capphi(c->grid.N), xi(nnz), xi1(nnz);
    std::vector<double> A(nnz);
    rc = dgv_export_A(ctx, &nnz, capphi.data(), A.data(), xi.data(), xi1.data());
    if (rc) return rc;
    for (int64_t k = 0; k < nnz; k++) {  // the file stores 1-based node indices
        xi[k] += 1;
        xi1[k] += 1;
    }
    std::string e = write_file(path, (int32_t)c->grid.N, nnz, capphi.data(), A.data(), xi.data(), xi1.data(),
                               max_subrecord ? max_subrecord : kMaxSubrecord);
    if (!e.empty()) return set_err(c, DGV_EINVAL, "write_A_file: " + e);
    return DGV_OK;
}
