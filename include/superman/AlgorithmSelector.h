// Chooses the permanent routine for a matrix — the reference's
// AlgorithmSelector<C,S>::selectAlgorithm (CommonFiles/AlgorithmSelector.h:
// 49-141), same rules on the GPU:
//  * algorithm "auto": dense (xregister_mshared) when n*sparsity/100 <= 6 or
//    the largest component has at most 41 (or n-3) vertices, otherwise the
//    sparse route (the reference's code-generation algorithms);
//  * any sparse-style algorithm, or a non-register algorithm on a matrix
//    below 30 % density, takes the sparse driver.
//  * "approximation" takes the sampling driver (gpuApproxSingleGPU).
// This library computes on one GPU only: mode=cpu and the multi-GPU modes
// are reported as unavailable (the reference's own error for modes it was
// not built with).
#pragma once

#include <stdexcept>

#include "GPUKernelWrappers.h"
#include "Matrix.h"
#include "Result.h"
#include "Settings.h"

template <class C, class S>
class AlgorithmSelector {
public:
    typedef Result (*Algorithm)(Matrix<S>* matrix, Settings* settings);

    static Algorithm selectAlgorithm(Matrix<S>* matrix, Settings* settings, unsigned biggestComponentSize)
    {
        if (settings->mode != SingleGPU)
            throw std::runtime_error(
                "The mode you want to calculate the permanent in is unavailable for launch. Terminating...\n");
        if (settings->algorithm == APPROXIMATION) return &gpuApproxSingleGPU<C, S>;
        if (settings->algorithm == AlgorithmEnds) {
            const bool dense = (matrix->nov * matrix->sparsity / 100 <= 6) || (biggestComponentSize <= 41) ||
                               ((int)biggestComponentSize <= matrix->nov - 3);
            settings->algorithm = dense ? XREGISTERMSHARED : REGEFFICIENTCODEGENERATION;
        }
        const ::Algorithm a = settings->algorithm;
        const bool sparse = a == NAIVECODEGENERATION || a == REGEFFICIENTCODEGENERATION ||
                            (a != XREGISTERMSHARED && a != XREGISTERMGLOBAL && matrix->sparsity < 30);
        return sparse ? &gpuSPSingleGPU<C, S> : &gpuDPSingleGPU<C, S>;
    }
};
