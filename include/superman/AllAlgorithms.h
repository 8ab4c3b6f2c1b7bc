// Umbrella header of the C++ mirror of the reference's API
// (Algorithms/AllAlgorithms.h): data contracts, reader, decomposition,
// selector and GPU drivers, all backed by libsupb200.
#pragma once

#include <complex>
#include <stdexcept>

#include "AlgorithmSelector.h"
#include "DecomposePerman.h"
#include "GPUKernelWrappers.h"
#include "IO.h"
#include "Matrix.h"
#include "Permanent.h"
#include "Result.h"
#include "Settings.h"
#include "SparseMatrix.h"
#include "dm.h"

// The reference's complexPerman (Algorithms/AllAlgorithms.h:93-110) on the GPU.
template <typename C, typename S>
void complexPerman(Matrix<std::complex<S>>* matrix, Settings* settings)
{
    if (settings->mode != SingleGPU)
        throw std::runtime_error("The mode you want to calculate the permanent in is unavailable for launch. Terminating...\n");
    gpuComputeComplex(matrix, settings);
}
