// faf_types.h -- plan types shared by host code and kernels.
#pragma once

#include <cuda_runtime.h>

namespace fafd {

constexpr int kMaxStages = 24;

struct Stage {
    int R;    // radix
    int p;    // product of the radices of the previous stages
    int tws;  // twiddle index stride into the n-point table: n / (p * R)
    int pad_;
};

// Per-size plan as passed to kernels.  The stage list lives in device memory
// (indexing a kernel-parameter array with a runtime stage counter would make
// the compiler copy the whole parameter block to local memory).
struct Shape {
    int n;               // transform length
    int ns;              // number of stages
    int T;               // threads per transform
    int plane;           // floats per shared-memory plane (padded)
    const Stage* st;     // device array of ns stages
};

}  // namespace fafd
