// fherma_abi.h -- the three C++ entry points the FHERMA harness binds for this challenge
// (fherma.toml:7-10: init = fherma_init, run = fherma_run, free = fherma_free), with the
// argument types of the platform header (fherma.h:8-48).
//
// The platform generates its own fherma.h; a build inside the platform defines
// POLYMULT_USE_PLATFORM_FHERMA_H and puts that header on the include path, so these
// functions bind to the platform's types.  Otherwise the types below are used: the same
// members in the same order (a Tensor is a shape vector plus a row-major data vector), which
// is what makes the three symbols link against the platform's main.cpp unchanged.
#pragma once

#ifdef POLYMULT_USE_PLATFORM_FHERMA_H
#include <fherma.h>
#else
#include <cstdint>
#include <vector>

namespace fherma {

template <class T>
struct Tensor {
    std::vector<int64_t> shape;
    std::vector<T> data;  // row-major
    int64_t count() const {
        int64_t n = 1;
        for (int64_t d : shape) n *= d;
        return n;
    }
};

struct Point {
    uint32_t N = 0;
    uint32_t W = 0;
    uint32_t L = 0;
    Tensor<uint32_t> q;  // L limbs
};

struct Inputs {
    Tensor<uint32_t> a;  // N x L
    Tensor<uint32_t> b;  // N x L
};

struct Outputs {
    Tensor<uint32_t> c;  // N x L
};

}  // namespace fherma

// Validates the point and prepares everything (tables, buffers, streams, warm-up);
// throws std::runtime_error on an invalid point or a CUDA failure.
void* fherma_init(const fherma::Point& p);
// c = a*b mod (X^N+1, q); throws std::runtime_error on a size mismatch or a failure.
fherma::Outputs fherma_run(void* state, const fherma::Inputs& in);
// Releases the state (nullptr accepted).
void fherma_free(void* state);
#endif
