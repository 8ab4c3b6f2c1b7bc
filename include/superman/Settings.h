// Run settings and their enums, field for field the reference's Settings
// (CommonFiles/Settings.h:36-102).  Unlike the reference, no mutable globals
// (avgN, sparse, printing) are shared between calls: whatever a driver needs
// travels in Settings or in the driver type.
#pragma once

#include <string>

enum Algorithm {
    XREGISTERMSHARED,
    XREGISTERMGLOBAL,
    XGLOBALMGLOBAL,
    XGLOBALMSHARED,
    XSHAREDMGLOBAL,
    XSHAREDMSHARED,
    NAIVECODEGENERATION,
    REGEFFICIENTCODEGENERATION,
    APPROXIMATION,
    AlgorithmEnds
};

enum Mode { CPU, SingleGPU, MultiGPU, MultiGPUMPI, ModeEnds };

enum Precision { DD, KAHAN, ARBITRARY, PrecisionEnds };

struct Settings {
    std::string filename;
    int PID = 2;
    std::string REPO_DIR;
    std::string pipe;
    Algorithm algorithm = AlgorithmEnds;  // AlgorithmEnds = "auto"
    Mode mode = SingleGPU;

    bool complex = false;
    bool binary = false;
    bool undirected = false;

    bool scaling = false;
    unsigned scalingIterationNo = 100;
    unsigned scaleInto = 2;

    unsigned arbitraryPrecision = 0;
    Precision calculationPrecision = KAHAN;

    int threadC = 1;

    int deviceID = 0;
    int gpuNum = 1;
    unsigned partition = 1;

    int rank = 0;
    int processorNum = 1;

    // Approximation (algorithm=approximation): number of samples (the
    // reference's NO_SAMPLES, Algorithms/GPU/GPUHelpers.cuh:39) and the seed
    // of the sample streams.  Keys approx_samples= and approx_seed=.
    unsigned long long approxSamples = 100000000ull;
    unsigned long long approxSeed = 1ull;
};
