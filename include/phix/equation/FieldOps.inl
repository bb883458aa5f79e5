// FieldOps.inl -- arithmetic on fields and terms (included by TermPW.inl):
// f1*f2, f1+f2, f1-f2, s*f, f+s, s-f, -f as pw terms; Term*Field, Term*Term,
// RHSExpr*... as composites that materialise each operand into scratch and
// multiply (the reference's include/equation/FieldOps.inl semantics).
#pragma once

namespace PhiX {
namespace detail {
// materialise an expression into a zeroed stored-size scratch buffer
void materialiseGPU(const RHSExpr& e, double* d_buf, std::size_t storedSize, ScratchPool& pool);
void materialiseGPU(const Term& t, double* d_buf, std::size_t storedSize, ScratchPool& pool);
void materialiseCPU(const RHSExpr& e, double* h_buf, std::size_t storedSize, ScratchPool& pool);
void materialiseCPU(const Term& t, double* h_buf, std::size_t storedSize, ScratchPool& pool);
const ScalarField* repField(const Term& t);
const ScalarField* repField(const RHSExpr& e);
Term timesField(const RHSExpr& lhs, const ScalarField& f, const ScalarField& layout);
Term timesExpr(const RHSExpr& a, const RHSExpr& b, const ScalarField& layout);
}  // namespace detail

inline Term operator*(const ScalarField& a, const ScalarField& b) {
    return pw(a, b, [] __host__ __device__(double x, double y) { return x * y; });
}
inline Term operator+(const ScalarField& a, const ScalarField& b) {
    return pw(a, b, [] __host__ __device__(double x, double y) { return x + y; });
}
inline Term operator-(const ScalarField& a, const ScalarField& b) {
    return pw(a, b, [] __host__ __device__(double x, double y) { return x - y; });
}
inline Term operator*(double s, const ScalarField& f) { return pw(f, [] __host__ __device__(double v) { return v; }, s); }
inline Term operator*(const ScalarField& f, double s) { return pw(f, [] __host__ __device__(double v) { return v; }, s); }
inline Term operator+(const ScalarField& f, double s) { return pw(f, [s] __host__ __device__(double v) { return v + s; }); }
inline Term operator+(double s, const ScalarField& f) { return pw(f, [s] __host__ __device__(double v) { return v + s; }); }
inline Term operator-(const ScalarField& f, double s) { return pw(f, [s] __host__ __device__(double v) { return v - s; }); }
inline Term operator-(double s, const ScalarField& f) { return pw(f, [s] __host__ __device__(double v) { return s - v; }); }
inline Term operator-(const ScalarField& f) { return pw(f, [] __host__ __device__(double v) { return -v; }); }

inline Term operator*(const Term& t, const ScalarField& f) { return detail::timesField(RHSExpr(t), f, *detail::repField(t)); }
inline Term operator*(const ScalarField& f, const Term& t) { return t * f; }
inline Term operator*(const Term& a, const Term& b) {
    return detail::timesExpr(RHSExpr(a), RHSExpr(b), *detail::repField(a));
}
inline Term operator*(const RHSExpr& e, const ScalarField& f) { return detail::timesField(e, f, *detail::repField(e)); }
inline Term operator*(const ScalarField& f, const RHSExpr& e) { return e * f; }
inline Term operator*(const RHSExpr& a, const Term& b) { return detail::timesExpr(a, RHSExpr(b), *detail::repField(a)); }
inline Term operator*(const Term& a, const RHSExpr& b) { return detail::timesExpr(RHSExpr(a), b, *detail::repField(a)); }
inline Term operator*(const RHSExpr& a, const RHSExpr& b) { return detail::timesExpr(a, b, *detail::repField(a)); }

inline VectorRHSExpr operator*(const Term& t, const VectorRHSExpr& v) {
    VectorRHSExpr out(v.nComponents());
    for (int c = 0; c < v.nComponents(); ++c) out[c] = RHSExpr(t * v[c]);
    return out;
}
inline VectorRHSExpr operator*(const VectorRHSExpr& v, const Term& t) { return t * v; }
inline VectorRHSExpr operator*(const ScalarField& f, const VectorRHSExpr& v) {
    VectorRHSExpr out(v.nComponents());
    for (int c = 0; c < v.nComponents(); ++c) out[c] = RHSExpr(f * v[c]);
    return out;
}
inline VectorRHSExpr operator*(const VectorRHSExpr& v, const ScalarField& f) { return f * v; }
inline VectorRHSExpr operator*(const RHSExpr& e, const VectorRHSExpr& v) {
    VectorRHSExpr out(v.nComponents());
    for (int c = 0; c < v.nComponents(); ++c) out[c] = RHSExpr(e * v[c]);
    return out;
}
inline VectorRHSExpr operator*(const VectorRHSExpr& v, const RHSExpr& e) { return e * v; }

}  // namespace PhiX
