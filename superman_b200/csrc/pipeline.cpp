// The reference's top-level flow (main.cpp:42-151) as C ABI entry points,
// built on the C++ mirror headers in include/superman/:
//   read / prune (IO::readMatrix, dm) -> components (findCCs) ->
//   AlgorithmSelector -> DecomposePerman -> GPU driver, per component,
//   permanent = product over components.
// Plus CPU-only hooks (reader, pruning, decomposition pieces) used by the
// host-logic tests.
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "AllAlgorithms.h"
#include "superman_b200.h"

void spb_set_error(const char* fmt, ...);

namespace {

Settings settings_from(const char* const* args, int nargs)
{
    Settings s;
    std::vector<std::string> store{"superman"};
    for (int i = 0; i < nargs; ++i) store.emplace_back(args[i] ? args[i] : "");
    bool hasFile = false;
    for (auto& a : store)
        if (a.rfind("filename=", 0) == 0) hasFile = true;
    if (!hasFile) store.emplace_back("filename=<memory>");
    std::vector<char*> argv;
    for (auto& a : store) argv.push_back(&a[0]);
    IO::readSettings(s, (int)argv.size(), argv.data());
    return s;
}

// Entries on no perfect matching removed in place, as IO::readMatrix does
// (IO/IO.h:477-508); the sparsity is updated.
void prune_in_place(Matrix<double>* matrix)
{
    const int n = matrix->nov;
    {
        std::vector<int> rptrs(n + 1, 0), cols;
        for (int r = 0; r < n; ++r) {
            for (int c = 0; c < n; ++c)
                if (matrix->mat[(size_t)r * n + c] != 0.0) cols.push_back(c);
            rptrs[r + 1] = (int)cols.size();
        }
        dm_prune(rptrs, cols, n);
        std::vector<double> kept((size_t)n * n, 0.0);
        for (int r = 0; r < n; ++r)
            for (int p = rptrs[r]; p < rptrs[r + 1]; ++p) kept[(size_t)r * n + cols[p]] = matrix->mat[(size_t)r * n + cols[p]];
        std::copy(kept.begin(), kept.end(), matrix->mat);
        matrix->sparsity = n ? 100.0 * rptrs[n] / ((double)n * n) : 0.0;
    }
}

// Component k of the pruned matrix as its own square block (main.cpp:91-101).
void component_block(const Matrix<double>* matrix, const std::vector<unsigned>& rows,
                     const std::vector<unsigned>& cols, Matrix<double>* block)
{
    const int n = matrix->nov;
    const unsigned m = (unsigned)rows.size();
    for (unsigned i = 0; i < m; ++i)
        for (unsigned j = 0; j < m; ++j) block->mat[(size_t)i * m + j] = matrix->mat[(size_t)rows[i] * n + cols[j]];
    block->sparsity = 100.0 * getNNZ(block) / ((double)m * m);
}

// main.cpp:63-110 on an in-memory matrix (the reader's pruning included).
void real_pipeline(Matrix<double>* matrix, Settings& settings, spb_pipeline_result* out)
{
    const int n = matrix->nov;
    prune_in_place(matrix);
    std::vector<std::vector<unsigned>> rc, cc;
    unsigned biggest = 0;
    findCCs(matrix, rc, cc, biggest);
    auto algorithm = AlgorithmSelector<double, double>::selectAlgorithm(matrix, &settings, biggest);
    g_decomposeStats = DecomposeStats{};
    Result result(0, n != 0 ? 1.0 : 0.0);
    for (size_t k = 0; k < rc.size(); ++k) {
        if (rc[k].size() != cc[k].size()) {
            result.permanent = 0;
            break;
        }
        Matrix<double> block((int)rc[k].size());
        component_block(matrix, rc[k], cc[k], &block);
        Result b = algorithm(&block, &settings);
        result.time += b.time;
        result.permanent *= b.permanent;
    }
    out->permanent = result.permanent;
    out->time_s = result.time;
    out->components = (int)rc.size();
    out->pieces = g_decomposeStats.pieces;
    out->avg_n = g_decomposeStats.pieces ? g_decomposeStats.sumN / g_decomposeStats.pieces : 0.0;
    out->avg_nnz = g_decomposeStats.pieces ? g_decomposeStats.sumNNZ / g_decomposeStats.pieces : 0.0;
    out->algorithm = settings.algorithm;
}

template <class F>
int guarded(F&& f)
{
    try {
        return f();
    } catch (const std::exception& e) {
        std::string msg = e.what();
        while (!msg.empty() && msg.back() == '\n') msg.pop_back();
        spb_set_error("%s", msg.c_str());
        if (msg.find("not square") != std::string::npos) return SPB_ERR_NOT_SQUARE;
        if (msg.find("could not be opened") != std::string::npos || msg.find("Matrix file") != std::string::npos)
            return SPB_ERR_IO;
        if (msg.find("superman_b200:") == 0) return SPB_ERR_CUDA;
        return SPB_ERR_INVALID;
    }
}

}  // namespace

extern "C" int spb_perm_pipeline(const double* a, int n, const char* const* args, int nargs,
                                 spb_pipeline_result* out)
{
    if (!out) return SPB_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    if (!a || n < 0) {
        spb_set_error("spb_perm_pipeline: null matrix or negative n");
        return out->status = SPB_ERR_INVALID;
    }
    return out->status = guarded([&] {
        Settings s = settings_from(args, nargs);
        Matrix<double> m(n);
        std::copy(a, a + (size_t)n * n, m.mat);
        real_pipeline(&m, s, out);
        return SPB_OK;
    });
}

extern "C" int spb_perm_file(const char* const* args, int nargs, spb_pipeline_result* out)
{
    if (!out) return SPB_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    return out->status = guarded([&] {
        Settings s = settings_from(args, nargs);
        if (s.complex) {
            std::unique_ptr<Matrix<std::complex<double>>> m(IO::readComplex<double>(s.filename, s));
            if (s.mode != SingleGPU)
                throw std::runtime_error("The mode you want to calculate the permanent in is unavailable for launch. Terminating...\n");
            ComplexResult r = gpuComplexPermanent(m.get(), &s);
            out->permanent = r.permanent.real();
            out->imag = r.permanent.imag();
            out->time_s = r.time;
            out->components = 1;
            out->pieces = 1;
            out->avg_n = m->nov;
            return SPB_OK;
        }
        std::unique_ptr<Matrix<double>> m(IO::readMatrix<double>(s.filename, s));
        real_pipeline(m.get(), s, out);
        return SPB_OK;
    });
}

extern "C" int spb_read_matrix(const char* path, int binary, int undirected, int is_complex, double* out,
                               int max_n, int* n_out, double* sparsity)
{
    if (!path || !n_out) return SPB_ERR_INVALID;
    return guarded([&] {
        Settings s;
        s.binary = binary != 0;
        s.undirected = undirected != 0;
        if (is_complex) {
            std::unique_ptr<Matrix<std::complex<double>>> m(IO::readComplex<double>(path, s));
            *n_out = m->nov;
            if (sparsity) *sparsity = m->sparsity;
            if (out && m->nov <= max_n)
                std::memcpy(out, m->mat, sizeof(double) * 2 * (size_t)m->nov * m->nov);
            return (out && m->nov > max_n) ? (int)SPB_ERR_INVALID : (int)SPB_OK;
        }
        std::unique_ptr<Matrix<double>> m(IO::readMatrix<double>(path, s));
        *n_out = m->nov;
        if (sparsity) *sparsity = m->sparsity;
        if (out && m->nov <= max_n) std::memcpy(out, m->mat, sizeof(double) * (size_t)m->nov * m->nov);
        return (out && m->nov > max_n) ? (int)SPB_ERR_INVALID : (int)SPB_OK;
    });
}

extern "C" int spb_dm_prune(const double* a, int n, double* out, int* has_perfect_matching)
{
    if (!a || !out || n < 0) return SPB_ERR_INVALID;
    std::vector<int> rptrs(n + 1, 0), cols;
    for (int r = 0; r < n; ++r) {
        for (int c = 0; c < n; ++c)
            if (a[(size_t)r * n + c] != 0.0) cols.push_back(c);
        rptrs[r + 1] = (int)cols.size();
    }
    const bool perfect = dm_prune(rptrs, cols, n);
    std::fill(out, out + (size_t)n * n, 0.0);
    for (int r = 0; r < n; ++r)
        for (int p = rptrs[r]; p < rptrs[r + 1]; ++p) out[(size_t)r * n + cols[p]] = a[(size_t)r * n + cols[p]];
    if (has_perfect_matching) *has_perfect_matching = perfect ? 1 : 0;
    return SPB_OK;
}

extern "C" int spb_decompose(const double* a, int n, int* count, int* sizes, double* data, int max_pieces,
                             size_t max_doubles)
{
    if (!a || !count || n < 0) return SPB_ERR_INVALID;
    return guarded([&] {
        Settings s;
        Matrix<double> m(n);
        std::copy(a, a + (size_t)n * n, m.mat);
        struct NoDriver : Permanent<double, double> {
            NoDriver(Matrix<double>* x, Settings st) : Permanent<double, double>(x, st) {}
            double permanentFunction() override { return 0.0; }
        };
        DecomposePerman<double, double, NoDriver> d(&m, s);
        std::vector<Matrix<double>*> ps = d.pieces();
        size_t need = 0;
        for (auto* p : ps) need += (size_t)p->nov * p->nov;
        *count = (int)ps.size();
        int st = SPB_OK;
        if (sizes && data && (int)ps.size() <= max_pieces && need <= max_doubles) {
            size_t off = 0;
            for (size_t k = 0; k < ps.size(); ++k) {
                sizes[k] = ps[k]->nov;
                std::memcpy(data + off, ps[k]->mat, sizeof(double) * (size_t)ps[k]->nov * ps[k]->nov);
                off += (size_t)ps[k]->nov * ps[k]->nov;
            }
        } else if (sizes || data) {
            st = SPB_ERR_INVALID;
        }
        for (auto* p : ps) delete p;
        return st;
    });
}

extern "C" int spb_plan_pieces(const double* a, int n, int* components, int* count, int* sizes,
                               int* piece_component, double* data, int max_pieces, size_t max_doubles)
{
    if (!a || !components || !count || n < 1) {
        spb_set_error("spb_plan_pieces: null argument or n < 1");
        return SPB_ERR_INVALID;
    }
    return guarded([&] {
        Settings s;
        Matrix<double> m(n);
        std::copy(a, a + (size_t)n * n, m.mat);
        prune_in_place(&m);
        std::vector<std::vector<unsigned>> rc, cc;
        unsigned biggest = 0;
        findCCs(&m, rc, cc, biggest);
        struct NoDriver : Permanent<double, double> {
            NoDriver(Matrix<double>* x, Settings st) : Permanent<double, double>(x, st) {}
            double permanentFunction() override { return 0.0; }
        };
        std::vector<std::unique_ptr<Matrix<double>>> ps;
        std::vector<int> owner;
        int ncomp = 0;
        for (size_t k = 0; k < rc.size(); ++k) {
            if (rc[k].size() != cc[k].size()) {  // structurally zero (main.cpp:86-90)
                ps.clear();
                owner.clear();
                ncomp = 1;
                break;
            }
            Matrix<double> block((int)rc[k].size());
            component_block(&m, rc[k], cc[k], &block);
            DecomposePerman<double, double, NoDriver> d(&block, s);
            for (Matrix<double>* p : d.pieces()) {
                ps.emplace_back(p);
                owner.push_back(ncomp);
            }
            ++ncomp;
        }
        *components = ncomp;
        *count = (int)ps.size();
        size_t need = 0;
        for (auto& p : ps) need += (size_t)p->nov * p->nov;
        if (!sizes && !piece_component && !data) return (int)SPB_OK;
        if (!sizes || !piece_component || !data || (int)ps.size() > max_pieces || need > max_doubles) {
            spb_set_error("spb_plan_pieces: %d pieces of %zu doubles do not fit the arrays (%d, %zu)",
                          (int)ps.size(), need, max_pieces, max_doubles);
            return (int)SPB_ERR_INVALID;
        }
        size_t off = 0;
        for (size_t k = 0; k < ps.size(); ++k) {
            sizes[k] = ps[k]->nov;
            piece_component[k] = owner[k];
            std::memcpy(data + off, ps[k]->mat, sizeof(double) * (size_t)ps[k]->nov * ps[k]->nov);
            off += (size_t)ps[k]->nov * ps[k]->nov;
        }
        return (int)SPB_OK;
    });
}

extern "C" int spb_reorder(const double* a, int n, const char* order, unsigned long long param, double* out)
{
    if (!a || !out || !order || n < 0) {
        spb_set_error("spb_reorder: null argument or negative n");
        return SPB_ERR_INVALID;
    }
    return guarded([&] {
        Matrix<double> m(n);
        std::copy(a, a + (size_t)n * n, m.mat);
        const std::string o(order);
        if (o == "colSort") IO::colSort(&m, param == 0);
        else if (o == "rowSort") IO::rowSort(&m, param == 0);
        else if (o == "skipOrder") IO::skipOrder(&m);
        else if (o == "UTOrder") IO::UTOrder(&m);
        else if (o == "colIndexMinimizationOrder") IO::colIndexMinimizationOrder(&m);
        else if (o == "alphaOrder") IO::alphaOrder(&m, (unsigned)(param ? param : 2));
        else if (o == "randomOrder") IO::randomOrder(&m, param);
        else throw std::runtime_error("spb_reorder: unknown order " + o);
        std::copy(m.mat, m.mat + (size_t)n * n, out);
        return (int)SPB_OK;
    });
}
