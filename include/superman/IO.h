// Matrix files, orderings, scaling and run settings — the reference's IO
// class (IO/IO.h): readMatrix (:403-515), readComplex (:517-596), the row
// and column orderings colSort / rowSort (:677-833), skipOrder (:598-679),
// colIndexMinimizationOrder (:891-924), UTOrder (:926-1002), alphaOrder
// (:1004-1071), randomOrder (:1073-1093) with applyPermutations
// (:1095-1112), scale (:109-161) and readSettings (:163-401), with the same
// file format and error messages.
//
// File format: optional '%' comment lines, a header "rows cols lines", then
// one "i j [value]" line per entry ("i j re im" for complex).  Indices are
// 1-based when the file name ends in ".mtx", 0-based otherwise; binary=true
// reads two columns and sets every listed entry to 1; undirected=true mirrors
// every entry; real matrices lose the entries that lie on no perfect matching
// (dm_prune) as in the reference.  Unlike the reference, an index outside the
// matrix is an error instead of an out-of-bounds write.
#pragma once

#include <algorithm>
#include <climits>
#include <cmath>
#include <complex>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "Helpers.h"
#include "Matrix.h"
#include "Settings.h"
#include "dm.h"

class IO {
public:
    static std::vector<std::string> split(const std::string& s, char delimiter)
    {
        std::vector<std::string> out;
        std::string tok;
        std::istringstream in(s);
        while (std::getline(in, tok, delimiter)) {
            size_t b = tok.find_first_not_of(" \t\r\n"), e = tok.find_last_not_of(" \t\r\n");
            out.push_back(b == std::string::npos ? std::string() : tok.substr(b, e - b + 1));
        }
        return out;
    }

    static bool isMTX(const std::string& filename)
    {
        auto parts = split(filename, '.');
        return !parts.empty() && parts.back() == "mtx";
    }

    template <class S>
    static Matrix<S>* readMatrix(const std::string& filename, Settings& settings)
    {
        std::ifstream file(filename);
        if (!file.is_open()) throw std::runtime_error("File could not be opened.\n");
        const bool mtx = isMTX(filename);
        int n = readHeader(file);
        std::vector<S> mat((size_t)n * n, S(0));
        int nnz = 0;
        int lines = pending_lines_;
        for (int it = 0; it < lines; ++it) {
            long i, j;
            S val = S(1);
            if (!(file >> i >> j)) throw std::runtime_error("Matrix file ended before all entries were read.\n");
            if (!settings.binary && !(file >> val)) throw std::runtime_error("Matrix file has a malformed entry.\n");
            if (val == S(0)) continue;
            if (mtx) { --i; --j; }
            checkIndex(i, j, n);
            mat[(size_t)i * n + j] = val;
            ++nnz;
            if (settings.undirected && i != j) {
                mat[(size_t)j * n + i] = val;
                ++nnz;
            }
        }
        // entries on no perfect matching are removed (they do not change the permanent)
        std::vector<int> rptrs(n + 1, 0), cols;
        for (int r = 0; r < n; ++r) {
            for (int c = 0; c < n; ++c)
                if (mat[(size_t)r * n + c] != S(0)) cols.push_back(c);
            rptrs[r + 1] = (int)cols.size();
        }
        dm_prune(rptrs, cols, n);
        auto* m = new Matrix<S>(n);
        for (int r = 0; r < n; ++r)
            for (int p = rptrs[r]; p < rptrs[r + 1]; ++p) m->mat[(size_t)r * n + cols[p]] = mat[(size_t)r * n + cols[p]];
        const int kept = rptrs[n];
        m->sparsity = n ? 100.0 * kept / ((double)n * n) : 0.0;
        (void)nnz;
        return m;
    }

    template <class S>
    static Matrix<std::complex<S>>* readComplex(const std::string& filename, Settings& settings)
    {
        std::ifstream file(filename);
        if (!file.is_open()) throw std::runtime_error("File could not be opened.\n");
        const bool mtx = isMTX(filename);
        int n = readHeader(file);
        int lines = pending_lines_;
        auto* m = new Matrix<std::complex<S>>(n);
        for (int it = 0; it < lines; ++it) {
            long i, j;
            S re, im;
            if (!(file >> i >> j >> re >> im)) throw std::runtime_error("Matrix file has a malformed entry.\n");
            if (mtx) { --i; --j; }
            checkIndex(i, j, n);
            m->mat[(size_t)i * n + j] = std::complex<S>(re, im);
            if (settings.undirected) m->mat[(size_t)j * n + i] = std::complex<S>(re, im);
        }
        const int nnz = settings.undirected ? 2 * lines : lines;
        m->sparsity = n ? 100.0 * nnz / ((double)n * n) : 0.0;
        return m;
    }

    // Columns reordered by ascending (or descending) nonzero count; ties keep
    // their original order.
    template <class S>
    static void colSort(Matrix<S>* m, bool ascending = true) { permuteByDegree(m, ascending, true); }

    template <class S>
    static void rowSort(Matrix<S>* m, bool ascending = true) { permuteByDegree(m, ascending, false); }

    // Moves row i to position rowTo[i] and column j to colTo[j] (IO/IO.h:1095-1112).
    template <class S>
    static void applyPermutations(Matrix<S>* m, const int* rowTo, const int* colTo)
    {
        const int n = m->nov;
        S* nm = new S[(size_t)n * n];
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) nm[(size_t)rowTo[i] * n + colTo[j]] = m->mat[(size_t)i * n + j];
        delete[] m->mat;
        m->mat = nm;
    }

    // Upper-triangular-leaning order for the register-efficient generated
    // kernels (IO/IO.h:926-1002): repeatedly take the column with the fewest
    // nonzeros in rows not yet placed, place it next, then place (in index
    // order) its rows not yet placed; rows never reached go last.
    template <class S>
    static void UTOrder(Matrix<S>* m)
    {
        const int n = m->nov;
        std::vector<int> rowTo(n), colTo(n);
        std::vector<long> open(n, 0);  // nonzeros of column j in unplaced rows; -1 once placed
        for (int j = 0; j < n; ++j) open[j] = getColNNZ(m, j);
        std::vector<char> placed(n, 0);
        int nextRow = 0;
        for (int step = 0; step < n; ++step) {
            int c = -1;
            for (int j = 0; j < n; ++j)
                if (open[j] >= 0 && (c < 0 || open[j] < open[c])) c = j;
            colTo[c] = step;
            open[c] = -1;
            for (int i = 0; i < n; ++i) {
                if (m->mat[(size_t)i * n + c] == S(0) || placed[i]) continue;
                placed[i] = 1;
                rowTo[i] = nextRow++;
                for (int j = 0; j < n; ++j)
                    if (open[j] >= 0 && m->mat[(size_t)i * n + j] != S(0)) --open[j];
            }
        }
        for (int i = 0; i < n; ++i)
            if (!placed[i]) rowTo[i] = nextRow++;
        applyPermutations(m, rowTo.data(), colTo.data());
    }

    // The reference's earlier form of the same order (IO/IO.h:598-679): the
    // same column choice and row placement, so the same result (rows never
    // reached, possible only with an empty row, go last here as in UTOrder).
    template <class S>
    static void skipOrder(Matrix<S>* m)
    {
        UTOrder(m);
    }

    // Renumbers the columns by first appearance, scanning rows in order
    // (IO/IO.h:891-924), so each row's columns lie as low as possible.
    template <class S>
    static void colIndexMinimizationOrder(Matrix<S>* m)
    {
        const int n = m->nov;
        std::vector<int> rowTo(n), colTo(n, -1);
        int next = 0;
        for (int i = 0; i < n; ++i) {
            rowTo[i] = i;
            for (int j = 0; j < n; ++j)
                if (m->mat[(size_t)i * n + j] != S(0) && colTo[j] < 0) colTo[j] = next++;
        }
        for (int j = 0; j < n; ++j)
            if (colTo[j] < 0) colTo[j] = next++;  // empty columns keep a place
        applyPermutations(m, rowTo.data(), colTo.data());
    }

    // Interleaves rows by degree (IO/IO.h:1004-1071): rows sorted by nonzero
    // count (descending unless `ascending`), then one row from the first
    // ceil(n/alpha) followed by alpha-1 from the end, repeatedly.  The
    // reference gives every row left over after the interleave the same
    // position (its final loop does not advance), which is not a
    // permutation; here they take the following positions.
    template <class S>
    static void alphaOrder(Matrix<S>* m, unsigned alpha, bool ascending = false)
    {
        const int n = m->nov;
        if (alpha < 1) alpha = 1;
        std::vector<int> order(n), deg(n), rowTo(n), colTo(n);
        for (int i = 0; i < n; ++i) {
            order[i] = i;
            deg[i] = getRowNNZ(m, i);
            colTo[i] = i;
        }
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return ascending ? deg[x] < deg[y] : deg[x] > deg[y]; });
        const int split = (int)std::ceil((double)n / alpha) - 1;
        int front = split, back = n - 1, cur = 0;
        while (split < back) {
            rowTo[order[front--]] = cur++;
            for (unsigned k = 0; k + 1 < alpha && split < back; ++k) rowTo[order[back--]] = cur++;
        }
        while (front >= 0) rowTo[order[front--]] = cur++;
        applyPermutations(m, rowTo.data(), colTo.data());
    }

    // Random row order (IO/IO.h:1073-1093); a fixed seed gives a repeatable
    // order, seed 0 a random one as in the reference.
    template <class S>
    static void randomOrder(Matrix<S>* m, unsigned long long seed = 0)
    {
        const int n = m->nov;
        std::vector<int> rowTo(n), colTo(n);
        for (int i = 0; i < n; ++i) rowTo[i] = colTo[i] = i;
        std::mt19937_64 g(seed ? seed : std::random_device{}());
        std::shuffle(rowTo.begin(), rowTo.end(), g);
        applyPermutations(m, rowTo.data(), colTo.data());
    }

    // Sinkhorn-style alternating row/column scaling towards line sums
    // settings.scaleInto, settings.scalingIterationNo rounds; the factors are
    // returned so the permanent can be rescaled afterwards.
    template <class C, class S>
    static void scale(Matrix<S>* m, const Settings& settings, ScalingCompact* sc)
    {
        const int n = m->nov;
        sc->rowScale = new double[n];
        sc->colScale = new double[n];
        std::fill(sc->rowScale, sc->rowScale + n, 1.0);
        std::fill(sc->colScale, sc->colScale + n, 1.0);
        for (unsigned it = 0; it < settings.scalingIterationNo; ++it) {
            for (int r = 0; r < n; ++r) {
                double s = 0;
                for (int c = 0; c < n; ++c) s += m->mat[(size_t)r * n + c] * sc->rowScale[r] * sc->colScale[c];
                if (s != 0) sc->rowScale[r] = double(settings.scaleInto) / s;
            }
            for (int c = 0; c < n; ++c) {
                double s = 0;
                for (int r = 0; r < n; ++r) s += m->mat[(size_t)r * n + c] * sc->rowScale[r] * sc->colScale[c];
                if (s != 0) sc->colScale[c] = double(settings.scaleInto) / s;
            }
        }
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) m->mat[(size_t)r * n + c] *= sc->rowScale[r] * sc->colScale[c];
    }

    // key=value arguments of the reference's command line (IO/IO.h:163-401).
    // pid and repo_dir belong to the reference's two-process launcher; they
    // are accepted and ignored here.
    static void readSettings(Settings& s, int argc, char* argv[])
    {
        bool haveFile = false;
        for (int a = 1; a < argc; ++a) {
            auto kv = split(argv[a], '=');
            if (kv.size() < 2) throw std::runtime_error(std::string("Malformed argument: ") + argv[a] + "\n");
            const std::string &k = kv[0], &v = kv[1];
            if (k == "filename") { s.filename = v; haveFile = true; }
            else if (k == "pid") s.PID = toInt(v, "pid");
            else if (k == "repo_dir") { s.REPO_DIR = v; s.pipe = v + "build/wrapper_pipe"; }
            else if (k == "algorithm") s.algorithm = parseAlgorithm(v);
            else if (k == "mode") {
                if (v == "cpu") { s.mode = CPU; s.algorithm = AlgorithmEnds; }
                else if (v == "single_gpu") s.mode = SingleGPU;
                else if (v == "multi_gpu") s.mode = MultiGPU;
                else if (v == "multi_gpu_mpi") s.mode = MultiGPUMPI;
                else throw std::runtime_error("UNKNOWN MODE: " + v + '\n');
            }
            else if (k == "thread_count") s.threadC = toInt(v, "thread_count");
            else if (k == "device_id") s.deviceID = toInt(v, "device_id");
            else if (k == "gpu_num") s.gpuNum = toInt(v, "gpu_num");
            else if (k == "complex") s.complex = v == "true";
            else if (k == "binary") s.binary = v == "true";
            else if (k == "undirected") s.undirected = v == "true";
            else if (k == "scaling") s.scaling = v == "true";
            else if (k == "scaling_iteration_no") s.scalingIterationNo = (unsigned)toInt(v, "scaling_iteration_no");
            else if (k == "approx_samples") s.approxSamples = toU64(v, "approx_samples");
            else if (k == "approx_seed") s.approxSeed = toU64(v, "approx_seed");
            else if (k == "scale_into") s.scaleInto = (unsigned)toInt(v, "scale_into");
            else if (k == "calculation_precision") {
                if (v == "kahan") s.calculationPrecision = KAHAN;
                else if (v == "dd") s.calculationPrecision = DD;
                else {
                    try {
                        s.arbitraryPrecision = (unsigned)std::stoul(v);
                        s.calculationPrecision = ARBITRARY;
                    } catch (const std::exception&) {
                        throw std::runtime_error("Calculation precision can either be kahan or dd or an arbitrary precision given as an unsigned integer!\n");
                    }
                }
            }
            else std::cerr << "UNKNOWN ARGUMENT: " << k << " - skipping it." << std::endl;
        }
        if (!haveFile)
            throw std::runtime_error("You are required to provide the absolute path of the matrix file that you want to calculate the matrix permanent for to the executable of this program!\n");
    }

    static Algorithm parseAlgorithm(const std::string& v)
    {
        static const std::pair<const char*, Algorithm> names[] = {
            {"auto", AlgorithmEnds}, {"xregister_mshared", XREGISTERMSHARED},
            {"xregister_mglobal", XREGISTERMGLOBAL}, {"xshared_mglobal", XSHAREDMGLOBAL},
            {"xshared_mshared", XSHAREDMSHARED}, {"xglobal_mglobal", XGLOBALMGLOBAL},
            {"xglobal_mshared", XGLOBALMSHARED}, {"naive_code_generation", NAIVECODEGENERATION},
            {"register_efficient_code_generation", REGEFFICIENTCODEGENERATION},
            {"approximation", APPROXIMATION}};
        for (auto& p : names)
            if (v == p.first) return p.second;
        throw std::runtime_error("UNKNOWN ALGORITHM: " + v + '\n');
    }

private:
    static inline thread_local int pending_lines_ = 0;

    static int readHeader(std::ifstream& file)
    {
        while (file.peek() == '%') file.ignore(1 << 20, '\n');
        long n = 0, m = 0, lines = 0;
        if (!(file >> n >> m >> lines)) throw std::runtime_error("Matrix file has no size header.\n");
        if (n != m)
            throw std::runtime_error("Your matrix is not square, and therefore the permanent of it is trivially equal to 0.");
        if (n < 0 || n > 1000000 || lines < 0) throw std::runtime_error("Matrix file header out of range.\n");
        pending_lines_ = (int)lines;
        return (int)n;
    }

    static void checkIndex(long i, long j, int n)
    {
        if (i < 0 || j < 0 || i >= n || j >= n)
            throw std::runtime_error("Matrix file has an entry outside the matrix (" + std::to_string(i) + ", " +
                                     std::to_string(j) + ").\n");
    }

    static int toInt(const std::string& v, const char* key)
    {
        try {
            return std::stoi(v);
        } catch (const std::exception&) {
            throw std::runtime_error(std::string("An integer value should be provided to the ") + key + " argument!\n");
        }
    }

    static unsigned long long toU64(const std::string& v, const char* key)
    {
        try {
            return std::stoull(v);
        } catch (const std::exception&) {
            throw std::runtime_error(std::string("An integer value should be provided to the ") + key + " argument!\n");
        }
    }

    template <class S>
    static void permuteByDegree(Matrix<S>* m, bool ascending, bool columns)
    {
        const int n = m->nov;
        std::vector<int> deg(n), order(n);
        for (int k = 0; k < n; ++k) {
            deg[k] = columns ? getColNNZ(m, k) : getRowNNZ(m, k);
            order[k] = k;
        }
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            return ascending ? deg[x] < deg[y] : deg[x] > deg[y];
        });
        S* nm = new S[(size_t)n * n];
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b)
                nm[(size_t)a * n + b] = columns ? m->mat[(size_t)a * n + order[b]] : m->mat[(size_t)order[a] * n + b];
        delete[] m->mat;
        m->mat = nm;
    }
};
