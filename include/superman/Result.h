// Result record {time, permanent} (CommonFiles/Result.h:29-37).
#pragma once

struct Result {
    Result(double t = 0, double p = 0) : time(t), permanent(p) {}
    double time;       // seconds spent computing
    double permanent;  // the permanent (NaN when the computation overflowed)
};
