// Command-line front end with the reference program's arguments and output
// (main.cpp:42-151, IO/IO.h:163-401):
//   superman filename=<f> [algorithm=auto|...] [mode=single_gpu]
//            [complex=true] [binary=true] [undirected=true]
//            [calculation_precision=kahan|dd] [scaling=true] [device_id=N]
// Prints "Submatrix count: ... - Average N: ... - Average NNZ: ..." and
// "Permanent: <value> - Computed in: <seconds> seconds." like the reference.
#include <cmath>
#include <complex>
#include <iomanip>
#include <iostream>
#include <limits>
#include <vector>

#include "superman_b200.h"

int main(int argc, char** argv)
{
    std::vector<const char*> args(argv + 1, argv + argc);
    spb_pipeline_result r;
    int st = spb_perm_file(args.data(), (int)args.size(), &r);
    if (st != SPB_OK) {
        std::cerr << spb_last_error() << std::endl;
        return 1;
    }
    bool cplx = false;
    for (const char* a : args)
        if (std::string(a) == "complex=true") cplx = true;
    std::cout << std::setprecision(std::numeric_limits<double>::max_digits10);
    if (!cplx)
        std::cout << "Submatrix count: " << r.pieces << " - Average N: " << r.avg_n << " - Average NNZ: " << r.avg_nnz
                  << std::endl;
    if (std::isnan(r.permanent) || std::isnan(r.imag)) {
        std::cout << "Permanent computation has overflowed. - Computed in: " << r.time_s << " seconds." << std::endl;
    } else if (cplx) {
        std::cout << "Permanent: " << std::complex<double>(r.permanent, r.imag) << " - Computed in: " << r.time_s
                  << " seconds." << std::endl;
    } else {
        std::cout << "Permanent: " << r.permanent << " - Computed in: " << r.time_s << " seconds." << std::endl;
    }
    return 0;
}
