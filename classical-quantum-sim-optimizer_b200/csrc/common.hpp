// Shared host-side types of the dqsim B200 statevector engine.
#pragma once

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace dq {

// Status codes of the C ABI (include/dqsim_sv.h).  Each maps to the Python
// exception class the reference raises for the same failure
// (src/monolithic/statevector/simulator.rs:204-372, src/codecs.rs:44-48).
enum Status : int {
    kOk = 0,
    kValueError = 1,     // parse / validation / query errors -> ValueError
    kMemoryError = 2,    // budget and allocation failures -> MemoryError
    kTypeError = 3,      // unknown option -> TypeError
    kRuntimeError = 4,   // profile write, nonfinite norm -> RuntimeError
    kNotImplemented = 5, // other backends -> NotImplementedError
    kCudaError = 6,      // device failure -> RuntimeError
};

struct Error : std::runtime_error {
    Status status;
    Error(Status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

[[noreturn]] inline void fail(Status s, const std::string& msg) { throw Error(s, msg); }

// Complex128 with num-complex 0.4 arithmetic:
//   (a*b).re = a.re*b.re - a.im*b.im, (a*b).im = a.re*b.im + a.im*b.re.
// Host files are compiled with -ffp-contract=off so no FMA changes rounding;
// this keeps fused 1q matrices bit-identical to the reference's.
struct cplx {
    double re = 0.0, im = 0.0;
    cplx() = default;
    constexpr cplx(double r, double i = 0.0) : re(r), im(i) {}
};
inline cplx operator*(cplx a, cplx b) { return cplx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
inline cplx operator+(cplx a, cplx b) { return cplx(a.re + b.re, a.im + b.im); }
inline cplx operator-(cplx a) { return cplx(-a.re, -a.im); }
inline bool operator==(cplx a, cplx b) { return a.re == b.re && a.im == b.im; }
inline bool operator!=(cplx a, cplx b) { return !(a == b); }

using Mat2 = std::array<std::array<cplx, 2>, 2>;

constexpr uint64_t kU64Max = ~uint64_t(0);
constexpr uint64_t kIsizeMax = (uint64_t(1) << 63) - 1;

}  // namespace dq
