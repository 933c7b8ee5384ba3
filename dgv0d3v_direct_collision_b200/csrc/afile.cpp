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
//
// A solution file (WriteSol_DGV / RestartSolutionDGV, readwrite.f90:1756-1800,
// 2389-2513) has the records (e_time, dt), (rkmts), (N) and one record with
// f, f1..f(rkmts-1), frhs1..frhs(rkmts-1): the solution, the previous
// solutions and right sides (divided by dt) of the multistep method.
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

// ---------------------------------------------------------------------------
// solution files

namespace {

// f may live on the host or the device: cudaMemcpyDefault infers the direction
std::string copy_any(double *dst, const double *src, size_t n)
{
    cudaError_t e = cudaMemcpy(dst, src, n * sizeof(double), cudaMemcpyDefault);
    return e == cudaSuccess ? "" : cudaGetErrorString(e);
}

// records of WriteSol_DGV: (e_time, dt), (rkmts), (N), then the (2 rkmts - 1)
// arrays of length N given as pieces
std::string write_sol(const char *path, int32_t N, int32_t rkmts, double e_time, double dt,
                      const std::vector<Piece> &arrays)
{
    if (rkmts < 1 || rkmts > 5) return "rkmts outside 1..5";
    File fp;
    fp.fp = fopen(path, "wb");
    if (!fp.fp) return std::string("cannot create ") + path;
    const double td[2] = {e_time, dt};
    const bool ok = write_record(fp.fp, {{td, 16}}, kMaxSubrecord) && write_record(fp.fp, {{&rkmts, 4}}, kMaxSubrecord) &&
                    write_record(fp.fp, {{&N, 4}}, kMaxSubrecord) && write_record(fp.fp, arrays, kMaxSubrecord);
    return ok ? "" : std::string("write failed for ") + path;
}

struct SolFile {
    double e_time = 0, dt = 0;
    int32_t rkmts = 0, N = 0;
    std::vector<unsigned char> arrays;  // f, f1..f(rkmts-1), frhs1..frhs(rkmts-1)
};

// RestartSolutionDGV's reads (readwrite.f90:2485-2507)
std::string read_sol(const char *path, SolFile &s)
{
    File fp;
    fp.fp = fopen(path, "rb");
    if (!fp.fp) return std::string("cannot open ") + path;
    std::vector<unsigned char> r1, r2, r3;
    std::string e = read_record(fp.fp, r1);
    if (e.empty()) e = read_record(fp.fp, r2);
    if (e.empty()) e = read_record(fp.fp, r3);
    if (e.empty()) e = read_record(fp.fp, s.arrays);
    if (!e.empty()) return e;
    if (r1.size() != 16 || r2.size() != 4 || r3.size() != 4) return "header records are not (e_time, dt), (rkmts), (N)";
    double td[2];
    std::memcpy(td, r1.data(), 16);
    std::memcpy(&s.rkmts, r2.data(), 4);
    std::memcpy(&s.N, r3.data(), 4);
    s.e_time = td[0];
    s.dt = td[1];
    if (s.rkmts < 1 || s.rkmts > 5) return "rkmts outside 1..5";
    if (s.N < 0) return "negative array length";
    if (s.arrays.size() != (size_t)(2 * s.rkmts - 1) * (size_t)s.N * sizeof(double))
        return "solution record length is not (2 rkmts - 1) N doubles";
    return "";
}

}  // namespace

extern "C" int dgv_write_solution_arrays(const char *path, int32_t N, int32_t rkmts, double e_time, double dt,
                                         const double *arrays)
{
    if (!path || N < 0 || (N > 0 && !arrays)) {
        g_file_err = "write_solution_arrays: bad arguments";
        return DGV_EINVAL;
    }
    g_file_err = write_sol(path, N, rkmts, e_time, dt, {{arrays, (size_t)(2 * rkmts - 1) * (size_t)N * sizeof(double)}});
    return g_file_err.empty() ? DGV_OK : DGV_EINVAL;
}

extern "C" int dgv_read_solution_arrays(const char *path, int32_t *N, int32_t *rkmts, double *e_time, double *dt,
                                        double *arrays)
{
    SolFile s;
    g_file_err = path ? read_sol(path, s) : "read_solution_arrays: NULL path";
    if (!g_file_err.empty()) return DGV_EINVAL;
    if (N) *N = s.N;
    if (rkmts) *rkmts = s.rkmts;
    if (e_time) *e_time = s.e_time;
    if (dt) *dt = s.dt;
    if (arrays) std::memcpy(arrays, s.arrays.data(), s.arrays.size());
    return DGV_OK;
}

extern "C" int dgv_write_solution(dgv_ctx *ctx, const char *path, const double *f, double e_time, double dt)
{
    if (!ctx) return DGV_EINVAL;
    Ctx *c = &ctx->c;
    if (!path || !f) return set_err(c, DGV_EINVAL, "write_solution: NULL argument");
    DGV_CUDA(c, cudaSetDevice(c->device));
    const size_t N = (size_t)c->grid.N;
    int order = 0;
    std::vector<double> frhs;
    int rc = ab_history_get(c, &order, frhs);
    if (rc) return rc;
    // before dgv_prepare_ab there is no multistep history: rkmts = 1
    const int rkmts = order > 0 ? order : 1;
    // f1..f4 are written as zeros: the multistep formulas never read them
    std::vector<double> fh(N), prev((size_t)(rkmts - 1) * N, 0.0);
    std::string e = copy_any(fh.data(), f, N);
    if (!e.empty()) return set_err(c, DGV_ECUDA, "write_solution: " + e);
    e = write_sol(path, (int32_t)N, rkmts, e_time, dt,
                  {{fh.data(), N * sizeof(double)},
                   {prev.data(), prev.size() * sizeof(double)},
                   {frhs.data(), frhs.size() * sizeof(double)}});
    if (!e.empty()) return set_err(c, DGV_EINVAL, "write_solution: " + e);
    return DGV_OK;
}

extern "C" int dgv_read_solution(dgv_ctx *ctx, const char *path, double *f, double *e_time, double *dt)
{
    if (!ctx) return DGV_EINVAL;
    Ctx *c = &ctx->c;
    if (!path || !f) return set_err(c, DGV_EINVAL, "read_solution: NULL argument");
    DGV_CUDA(c, cudaSetDevice(c->device));
    SolFile s;
    std::string e = read_sol(path, s);
    if (!e.empty()) return set_err(c, DGV_EINVAL, std::string("read_solution: ") + path + ": " + e);
    const size_t N = (size_t)c->grid.N;
    if ((size_t)s.N != N) return set_err(c, DGV_EINVAL, "read_solution: array length differs from the grid's N");
    const double *arr = reinterpret_cast<const double *>(s.arrays.data());
    e = copy_any(f, arr, N);
    if (!e.empty()) return set_err(c, DGV_ECUDA, "read_solution: " + e);
    int rc = ab_history_set(c, s.rkmts, arr + (size_t)s.rkmts * N);  // after f, f1..f(rkmts-1)
    if (rc) return rc;
    if (e_time) *e_time = s.e_time;
    if (dt) *dt = s.dt;
    return DGV_OK;
}
