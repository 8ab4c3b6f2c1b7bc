// GPU drivers and the wrapper functions the algorithm selector hands out —
// the reference's gpuDPSingleGPU / gpuSPSingleGPU
// (Algorithms/GPU/GPUKernelWrappers.h:34-57, .cu:208-268) and
// gpuComputeComplex (Algorithms/Complex/gpuComputeComplex.cuh:33), here
// backed by the C ABI of libsupb200 (include/superman_b200.h).
//
//  * spbDenseSingleGPU<C,S>  the dense driver (a Permanent): the whole-GPU
//    Nijenhuis-Wilf walk; calculationPrecision DD selects the double-double
//    re-evaluation of dominant terms, KAHAN the FP64 walk.
//  * spbSparseSingleGPU<C,S> the sparse driver: orders the columns by
//    ascending degree and builds the CSR/CSC view as the reference's sparse
//    drivers do (CommonFiles/Permanent.h:82-87), then hands the CSC arrays to
//    spb_perm_sparse_f64 (row-compacted walk when its cost model wins).
//  * binary=true on a 0/1 matrix computes the exact integer permanent.
#pragma once

#include <complex>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <vector>

#include "DecomposePerman.h"
#include "Helpers.h"
#include "IO.h"
#include "Matrix.h"
#include "Permanent.h"
#include "Result.h"
#include "Settings.h"
#include "SparseMatrix.h"
#include "superman_b200.h"

namespace spb_detail {

inline spb_options options_from(const Settings& s)
{
    spb_options o;
    spb_default_options(&o);
    o.device = s.deviceID;
    o.precision = s.calculationPrecision == DD ? SPB_PREC_DD : SPB_PREC_FP64;
    return o;
}

inline void check(int st)
{
    if (st != SPB_OK) throw std::runtime_error(std::string("superman_b200: ") + spb_last_error() + "\n");
}

template <class S>
inline bool is01(const Matrix<S>* m)
{
    for (size_t i = 0; i < (size_t)m->nov * m->nov; ++i)
        if (m->mat[i] != S(0) && m->mat[i] != S(1)) return false;
    return true;
}

template <class S>
inline double dense_permanent(const Matrix<S>* m, const Settings& s)
{
    const int n = m->nov;
    if (n == 0) return 1.0;
    spb_options o = options_from(s);
    spb_result r;
    if (s.binary && is01(m)) {
        std::vector<uint8_t> b((size_t)n * n);
        for (size_t i = 0; i < b.size(); ++i) b[i] = m->mat[i] != S(0);
        uint32_t limbs[10];
        check(spb_perm_binary(b.data(), n, &o, limbs, &r));
        return r.value;
    }
    std::vector<double> a(m->mat, m->mat + (size_t)n * n);
    check(spb_perm_dense_f64(a.data(), n, &o, &r));
    return r.value + r.value_lo;
}

// The sparse driver's permanent: the compressed-column arrays of the
// SparseMatrix go to spb_perm_sparse_f64 (row-compacted walk when it pays).
template <class S>
inline double sparse_permanent(const SparseMatrix<S>* m, const Settings& s)
{
    const int n = m->nov;
    if (n == 0) return 1.0;
    if (s.binary && is01(m)) return dense_permanent(m, s);
    spb_options o = options_from(s);
    spb_result r;
    std::vector<double> vals(m->cvals, m->cvals + m->cptrs[n]);
    check(spb_perm_sparse_f64(m->cptrs, m->rows, vals.data(), n, &o, &r));
    return r.value + r.value_lo;
}

}  // namespace spb_detail

template <class C, class S>
class spbDenseSingleGPU : public Permanent<C, S> {
public:
    spbDenseSingleGPU(Matrix<S>* matrix, Settings settings) : Permanent<C, S>(matrix, settings) {}
    double permanentFunction() final { return spb_detail::dense_permanent(this->m_Matrix, this->m_Settings); }
};

template <class C, class S>
class spbSparseSingleGPU : public Permanent<C, S> {
public:
    spbSparseSingleGPU(Matrix<S>* matrix, Settings settings) : Permanent<C, S>(matrix, settings) {}
    double permanentFunction() final
    {
        if (auto* sp = dynamic_cast<SparseMatrix<S>*>(this->m_Matrix))
            return spb_detail::sparse_permanent(sp, this->m_Settings);
        return spb_detail::dense_permanent(this->m_Matrix, this->m_Settings);
    }

protected:
    void prepare() override
    {
        IO::colSort(this->m_Matrix);
        this->m_Matrix = new SparseMatrix<S>(this->m_Matrix, getNNZ(this->m_Matrix));
    }
};

// Sampling driver, the reference's aspSingleGPU (Algorithms/GPU/Sparse/
// aspSingleGPU.cuh:45-165): rows sorted by degree and the sparse layout
// built as the reference's Permanent::computePermanent does for the
// approximation (CommonFiles/Permanent.h:76-81), then spb_perm_approx on the
// pattern.  Sample count and seed: Settings::approxSamples (default 1e8, the
// reference's NO_SAMPLES) and Settings::approxSeed.
template <class C, class S>
class spbApproxSingleGPU : public Permanent<C, S> {
public:
    spbApproxSingleGPU(Matrix<S>* matrix, Settings settings) : Permanent<C, S>(matrix, settings) {}
    double permanentFunction() final
    {
        auto* sp = dynamic_cast<SparseMatrix<S>*>(this->m_Matrix);
        if (!sp) throw std::runtime_error("superman_b200: the approximation driver needs its sparse layout\n");
        spb_options o = spb_detail::options_from(this->m_Settings);
        spb_result r;
        spb_detail::check(spb_perm_approx(sp->cptrs, sp->rows, sp->nov, this->m_Settings.approxSamples,
                                          this->m_Settings.approxSeed, &o, &r));
        return r.value;
    }

protected:
    void prepare() override
    {
        IO::rowSort(this->m_Matrix);
        this->m_Matrix = new SparseMatrix<S>(this->m_Matrix, getNNZ(this->m_Matrix));
    }
};

template <class C, class S>
Result gpuApproxSingleGPU(Matrix<S>* matrix, Settings* settings)
{
    DecomposePerman<C, S, spbApproxSingleGPU<C, S>> d(matrix, *settings);
    return d.computePermanentRecursively();
}

template <class C, class S>
Result gpuDPSingleGPU(Matrix<S>* matrix, Settings* settings)
{
    DecomposePerman<C, S, spbDenseSingleGPU<C, S>> d(matrix, *settings);
    return d.computePermanentRecursively();
}

template <class C, class S>
Result gpuSPSingleGPU(Matrix<S>* matrix, Settings* settings)
{
    DecomposePerman<C, S, spbSparseSingleGPU<C, S>> d(matrix, *settings);
    return d.computePermanentRecursively();
}

// Complex permanent with its value returned (the reference only prints it).
struct ComplexResult {
    double time;
    std::complex<double> permanent;
};

inline ComplexResult gpuComplexPermanent(const Matrix<std::complex<double>>* matrix, const Settings* settings)
{
    spb_options o = spb_detail::options_from(*settings);
    spb_result r;
    spb_detail::check(spb_perm_dense_c128(reinterpret_cast<const double*>(matrix->mat), matrix->nov, &o, &r));
    return {r.elapsed_s, std::complex<double>(r.value + r.value_lo, r.imag + r.imag_lo)};
}

// Same output as the reference (Algorithms/Complex/gpuComputeComplex.cu:396-417).
inline void gpuComputeComplex(Matrix<std::complex<double>>* matrix, Settings* settings)
{
    ComplexResult r = gpuComplexPermanent(matrix, settings);
    std::stringstream s;
    if (std::isnan(r.permanent.real()) || std::isnan(r.permanent.imag()))
        s << "Permanent computation has overflowed." << " - Computed in: " << r.time << " seconds." << std::endl;
    else
        s << "Permanent: " << std::setprecision(17) << r.permanent << " - Computed in: " << r.time << " seconds."
          << std::endl;
    if (settings->rank == 0) std::cout << s.str() << std::flush;
}
