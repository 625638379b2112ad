// ref_shim.cpp -- C entry points over the reference's own fherma_init / fherma_run /
// fherma_free.  TEST INFRASTRUCTURE ONLY.
//
// Compiled (by oracle/Makefile) together with the UNMODIFIED reference sources, solve.cu
// built as plain C++ against the reference's CPU emulator pm_emu.h exactly as
// tests/run_emu.sh:10-12 builds it.  The result, oracle/_ref/libref_emu.so, is the
// reference's CPU path: the checker for parity tests and the timed reference arm of
// bench.py.  fherma.h comes from the reference tree at build time (-I<reference>).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <stdexcept>

#include "fherma.h"

namespace {
void put_error(char* err, int errlen, const char* what) {
    if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "%s", what);
}
}  // namespace

extern "C" {

void* ref_init(uint32_t N, uint32_t W, uint32_t L, const uint32_t* q, char* err, int errlen) {
    try {
        fherma::Point pt;
        pt.N = N;
        pt.W = W;
        pt.L = L;
        pt.q.shape = {static_cast<int64_t>(L)};
        pt.q.data.assign(q, q + L);
        return fherma_init(pt);
    } catch (const std::exception& e) {
        put_error(err, errlen, e.what());
    } catch (...) {
        put_error(err, errlen, "unknown exception");
    }
    return nullptr;
}

int ref_run(void* state, uint32_t N, uint32_t L, const uint32_t* a, const uint32_t* b, uint32_t* c,
            char* err, int errlen) {
    try {
        fherma::Inputs in;
        const size_t words = (size_t)N * L;
        in.a.shape = {static_cast<int64_t>(N), static_cast<int64_t>(L)};
        in.b.shape = in.a.shape;
        in.a.data.assign(a, a + words);
        in.b.data.assign(b, b + words);
        fherma::Outputs out = fherma_run(state, in);
        if (out.c.data.size() != words) throw std::runtime_error("reference returned a wrong-sized result");
        std::memcpy(c, out.c.data.data(), words * 4);
        return 0;
    } catch (const std::exception& e) {
        put_error(err, errlen, e.what());
    } catch (...) {
        put_error(err, errlen, "unknown exception");
    }
    return -1;
}

void ref_free(void* state) { fherma_free(state); }

}  // extern "C"
